// liar_gpu.cu -- context, mesh and trace entry points of the C ABI declared in include/liar_gpu.h.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include "../../include/liar_gpu.h"
#include "ctx.h"
#include "qbvh.h"
#include "traverse.cuh"

using namespace liar_gpu;

struct liar_gpu_mesh {
    int device = -1;
    QNode* d_nodes = nullptr;
    QTri* d_tris = nullptr;
    liar_mesh_stats stats{};
};

namespace liar_gpu {

int ctx_fail(liar_gpu_ctx* ctx, int code, const char* fmt, ...) {
    if (ctx) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        std::vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        ctx->err = buf;
    }
    return code;
}

int ctx_cuda(liar_gpu_ctx* ctx, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return LIAR_OK;
    return ctx_fail(ctx, e == cudaErrorMemoryAllocation ? LIAR_ERR_OOM : LIAR_ERR_CUDA, "%s: %s", what,
                    cudaGetErrorString(e));
}

int ctx_activate(liar_gpu_ctx* ctx) {
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != ctx->device) return ctx_cuda(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    return LIAR_OK;
}

int ctx_grow(liar_gpu_ctx* ctx, void** buf, size_t* cap, size_t bytes, const char* what) {
    if (*cap >= bytes) return LIAR_OK;
    if (*buf) cudaFree(*buf);
    *buf = nullptr;
    *cap = 0;
    size_t want = bytes + bytes / 4;
    cudaError_t e = cudaMalloc(buf, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return ctx_cuda(ctx, e, what);
    }
    *cap = want;
    return LIAR_OK;
}

}  // namespace liar_gpu

// ------------------------------------------------------------------------------------------------
// trace launch

namespace {

template <bool ANY, int S, int BLOCK, bool COUNT>
int launch_trace_t(liar_gpu_ctx* ctx, const liar_gpu_mesh* m, const liar_ray* d_rays, uint32_t n, liar_hit* d_hits,
                   TraceCounters* d_counters, cudaStream_t st, uint32_t* d_counter, uint32_t* d_status,
                   const uint32_t* n_dev) {
    auto kern = trace_kernel<ANY, S, BLOCK, COUNT>;
    const size_t smem = (size_t)S * BLOCK * 8;
    int& per_sm = ctx->occupancy[(const void*)kern];
    if (per_sm == 0) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "set trace shared memory");
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BLOCK, smem);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "occupancy query");
        if (per_sm <= 0) per_sm = 1;
    }
    const uint64_t needed_blocks = ((uint64_t)n + BLOCK - 1) / BLOCK;
    uint64_t blocks = (uint64_t)ctx->num_sms * per_sm;
    if (blocks > needed_blocks) blocks = needed_blocks;
    if (blocks == 0) blocks = 1;
    cudaError_t e = cudaMemsetAsync(d_counter, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "reset work counter");
    const uint32_t batch = trace_batch(n, (uint32_t)blocks * (BLOCK / 32));
    kern<<<(unsigned)blocks, BLOCK, smem, st>>>(m->d_nodes, m->d_tris, d_rays, d_hits, n, d_counter, d_status,
                                             d_counters, batch, n_dev);
    return ctx_cuda(ctx, cudaGetLastError(), "trace kernel launch");
}

template <int S, int BLOCK>
int launch_trace_sb(liar_gpu_ctx* ctx, const liar_gpu_mesh* m, const liar_ray* d_rays, uint32_t n, liar_hit* d_hits,
                    int any_hit, TraceCounters* d_counters, cudaStream_t st, uint32_t* d_counter, uint32_t* d_status,
                    const uint32_t* n_dev) {
    const bool cnt = d_counters != nullptr;
    if (any_hit)
        return cnt ? launch_trace_t<true, S, BLOCK, true>(ctx, m, d_rays, n, d_hits, d_counters, st, d_counter, d_status, n_dev)
                   : launch_trace_t<true, S, BLOCK, false>(ctx, m, d_rays, n, d_hits, d_counters, st, d_counter, d_status, n_dev);
    return cnt ? launch_trace_t<false, S, BLOCK, true>(ctx, m, d_rays, n, d_hits, d_counters, st, d_counter, d_status, n_dev)
               : launch_trace_t<false, S, BLOCK, false>(ctx, m, d_rays, n, d_hits, d_counters, st, d_counter, d_status, n_dev);
}

int launch_trace(liar_gpu_ctx* ctx, const liar_gpu_mesh* m, const liar_ray* d_rays, size_t n_rays, liar_hit* d_hits,
                 int any_hit, TraceCounters* d_counters, cudaStream_t st, uint32_t* d_counter, uint32_t* d_status,
                 const uint32_t* n_dev = nullptr) {
    if (n_rays == 0) return LIAR_OK;
    // the work counter of the persistent warps overshoots n by BATCH per warp; 2^31 keeps it far from wrapping
    if (n_rays > (1ull << 31)) return ctx_fail(ctx, LIAR_ERR_INVALID, "too many rays in one call (limit 2^31)");
    if (((uintptr_t)d_rays & 15) || ((uintptr_t)d_hits & 7))
        return ctx_fail(ctx, LIAR_ERR_INVALID, "ray buffer must be 16-byte aligned and hit buffer 8-byte aligned");
    const uint32_t need = m->stats.stack_needed;
    if (need > (uint32_t)kTraceStackTotal)
        return ctx_fail(ctx, LIAR_ERR_STACK, "tree needs %u stack entries, more than the %d the kernels hold", need,
                        kTraceStackTotal);
    const uint32_t n = (uint32_t)n_rays;
    const int s = ctx->trace_cfg.smem_stack, b = ctx->trace_cfg.block_size;
#define LIAR_TRACE_CASE(S_, B_) \
    if (s == S_ && b == B_) return launch_trace_sb<S_, B_>(ctx, m, d_rays, n, d_hits, any_hit, d_counters, st, d_counter, d_status, n_dev);
    LIAR_TRACE_CASE(8, 128)
    LIAR_TRACE_CASE(16, 128)
    LIAR_TRACE_CASE(24, 128)
    LIAR_TRACE_CASE(8, 256)
    LIAR_TRACE_CASE(16, 256)
#undef LIAR_TRACE_CASE
    return ctx_fail(ctx, LIAR_ERR_INVALID, "no trace kernel for block %d, shared stack %d", b, s);
}

cudaStream_t pick_stream(liar_gpu_ctx* ctx, void* stream) {
    if (stream) return (cudaStream_t)stream;
    return ctx->stream;
}

}  // namespace

namespace liar_gpu {
// entry for the other subsystems of the library (renderer, photon tracer): one launch on a
// device ray buffer with the context's launch shape and the given work-counter word
int trace_mesh_internal(liar_gpu_ctx* ctx, const liar_gpu_mesh* mesh, const liar_ray* d_rays, size_t n,
                        liar_hit* d_hits, int any_hit, cudaStream_t st, int counter_word, const uint32_t* n_dev) {
    return launch_trace(ctx, mesh, d_rays, n, d_hits, any_hit, nullptr, st, ctx->d_scratch + counter_word,
                        ctx->d_scratch + kStatusWord, n_dev);
}
}  // namespace liar_gpu

// ------------------------------------------------------------------------------------------------
// context

extern "C" int liar_gpu_abi_version(void) { return LIAR_GPU_ABI_VERSION; }

extern "C" int liar_gpu_create(liar_gpu_ctx** out, int device) {
    if (!out) return LIAR_ERR_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return LIAR_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= n) return LIAR_ERR_INVALID;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return LIAR_ERR_CUDA;
    if (prop.major != 10) return LIAR_ERR_NO_DEVICE;  // built for sm_100a only
    liar_gpu_ctx* ctx = new (std::nothrow) liar_gpu_ctx();
    if (!ctx) return LIAR_ERR_OOM;
    ctx->device = device;
    ctx->num_sms = prop.multiProcessorCount;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc((void**)&ctx->d_scratch, kScratchWords * sizeof(uint32_t)) != cudaSuccess ||
        cudaMemset(ctx->d_scratch, 0, kScratchWords * sizeof(uint32_t)) != cudaSuccess) {
        cudaGetLastError();
        liar_gpu_destroy(ctx);
        return LIAR_ERR_CUDA;
    }
    ctx->stream = ctx->own_stream;
    *out = ctx;
    return LIAR_OK;
}

extern "C" void liar_gpu_destroy(liar_gpu_ctx* ctx) {
    if (!ctx) return;
    int cur = -1;
    cudaGetDevice(&cur);
    cudaSetDevice(ctx->device);
    if (ctx->own_stream) cudaStreamSynchronize(ctx->own_stream);
    ctx->release_extensions();
    if (ctx->d_rays) cudaFree(ctx->d_rays);
    if (ctx->d_hits) cudaFree(ctx->d_hits);
    if (ctx->d_scratch) cudaFree(ctx->d_scratch);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    if (cur >= 0) cudaSetDevice(cur);
    delete ctx;
}

extern "C" const char* liar_gpu_last_error(const liar_gpu_ctx* ctx) {
    if (!ctx) return "null context";
    return ctx->err.c_str();
}

extern "C" int liar_gpu_set_stream(liar_gpu_ctx* ctx, void* stream) {
    if (!ctx) return LIAR_ERR_INVALID;
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return LIAR_OK;
}

extern "C" int liar_gpu_synchronize(liar_gpu_ctx* ctx) {
    if (!ctx) return LIAR_ERR_INVALID;
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    rc = ctx_cuda(ctx, cudaStreamSynchronize(ctx->stream), "stream synchronize");
    if (rc) return rc;
    return ctx_check_status(ctx);
}

namespace liar_gpu {

int ctx_check_status(liar_gpu_ctx* ctx) {
    uint32_t status = 0;
    cudaError_t e = cudaMemcpy(&status, ctx->d_scratch + kStatusWord, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "read device status");
    if (status == 0) return LIAR_OK;
    cudaMemset(ctx->d_scratch + kStatusWord, 0, sizeof(uint32_t));
    if (status & STATUS_STACK_OVERFLOW)
        return ctx_fail(ctx, LIAR_ERR_STACK, "device traversal stack overflowed (status 0x%x)", status);
    if (status & kStatusTimeout) return ctx_fail(ctx, LIAR_ERR_TIMEOUT, "a bounded device wait gave up (status 0x%x)", status);
    return ctx_fail(ctx, LIAR_ERR_CUDA, "device reported status 0x%x", status);
}

int ctx_cancelled(liar_gpu_ctx* ctx, cudaStream_t st) {
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "cancel: wait for the queued work");
    const int rc = ctx_check_status(ctx);  // a device error of the finished work takes precedence
    if (rc) return rc;
    return ctx_fail(ctx, LIAR_ERR_CANCELLED, "render cancelled by the cancel flag");
}

}  // namespace liar_gpu

// ------------------------------------------------------------------------------------------------
// meshes

extern "C" int liar_gpu_mesh_build(liar_gpu_ctx* ctx, const float* vertices, size_t n_vertices,
                                   const uint32_t* triangles, size_t n_triangles, const liar_build_opts* opts,
                                   liar_gpu_mesh** out) {
    if (!ctx || !out) return LIAR_ERR_INVALID;
    *out = nullptr;
    if (!vertices || !triangles) return ctx_fail(ctx, LIAR_ERR_INVALID, "null vertex or triangle array");
    return liar_gpu::mesh_build_with_spheres(ctx, vertices, n_vertices, triangles, n_triangles, nullptr, 0, opts, out);
}

// the tree over a scene's triangles and analytic spheres (sphere k is primitive n_triangles + k)
int liar_gpu::mesh_build_with_spheres(liar_gpu_ctx* ctx, const float* vertices, size_t n_vertices,
                                      const uint32_t* triangles, size_t n_triangles, const float* spheres,
                                      size_t n_spheres, const liar_build_opts* opts, liar_gpu_mesh** out) {
    if (!ctx || !out) return LIAR_ERR_INVALID;
    *out = nullptr;
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    BuildOptions bo;
    if (opts) {
        if (opts->max_leaf_size) bo.max_leaf_size = opts->max_leaf_size;
        if (opts->sah_bins) bo.sah_bins = opts->sah_bins;
        if (opts->traversal_cost > 0) bo.traversal_cost = opts->traversal_cost;
        bo.threads = opts->threads;
    }
    const auto t0 = std::chrono::steady_clock::now();
    QBVHHost q;
    char msg[256] = {0};
    rc = build_qbvh(vertices, n_vertices, triangles, n_triangles, spheres, n_spheres, bo, q, msg, sizeof(msg));
    if (rc) return ctx_fail(ctx, rc, "mesh build: %s", msg);
    const auto t1 = std::chrono::steady_clock::now();
    liar_gpu_mesh* m = new (std::nothrow) liar_gpu_mesh();
    if (!m) {
        free_qbvh(q);
        return ctx_fail(ctx, LIAR_ERR_OOM, "host allocation");
    }
    m->device = ctx->device;
    const size_t nb = q.n_nodes * sizeof(QNode), tb = q.n_tris * sizeof(QTri);
    cudaError_t e = cudaMalloc((void**)&m->d_nodes, nb);
    if (e == cudaSuccess) e = cudaMalloc((void**)&m->d_tris, tb);
    if (e == cudaSuccess) e = cudaMemcpy(m->d_nodes, q.nodes, nb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(m->d_tris, q.tris, tb, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaGetLastError();
        free_qbvh(q);
        liar_gpu_mesh_destroy(m);
        return ctx_cuda(ctx, e, "mesh upload");
    }
    m->stats.n_triangles = q.n_tris;
    m->stats.n_nodes = q.n_nodes;
    m->stats.n_leaves = q.n_leaves;
    m->stats.max_depth = q.max_depth;
    m->stats.stack_needed = q.stack_needed;
    m->stats.sah_cost = q.sah_cost;
    m->stats.device_bytes = nb + tb;
    m->stats.build_seconds = std::chrono::duration<double>(t1 - t0).count();
    free_qbvh(q);
    *out = m;
    return LIAR_OK;
}

extern "C" void liar_gpu_mesh_destroy(liar_gpu_mesh* m) {
    if (!m) return;
    int cur = -1;
    cudaGetDevice(&cur);
    if (m->device >= 0) cudaSetDevice(m->device);
    if (m->d_nodes) cudaFree(m->d_nodes);
    if (m->d_tris) cudaFree(m->d_tris);
    if (cur >= 0) cudaSetDevice(cur);
    delete m;
}

extern "C" int liar_gpu_mesh_stats(const liar_gpu_mesh* m, liar_mesh_stats* out) {
    if (!m || !out) return LIAR_ERR_INVALID;
    *out = m->stats;
    return LIAR_OK;
}

namespace liar_gpu {
const QNode* mesh_nodes(const liar_gpu_mesh* m) { return m->d_nodes; }
const QTri* mesh_tris(const liar_gpu_mesh* m) { return m->d_tris; }
uint32_t mesh_stack_needed(const liar_gpu_mesh* m) { return m->stats.stack_needed; }
int mesh_device(const liar_gpu_mesh* m) { return m->device; }
}  // namespace liar_gpu

// ------------------------------------------------------------------------------------------------
// tracing

extern "C" int liar_gpu_trace_device(liar_gpu_ctx* ctx, const liar_gpu_mesh* mesh, const liar_ray* d_rays,
                                     size_t n_rays, liar_hit* d_hits, int any_hit, void* stream) {
    if (!ctx) return LIAR_ERR_INVALID;
    if (!mesh || (n_rays && (!d_rays || !d_hits))) return ctx_fail(ctx, LIAR_ERR_INVALID, "null mesh or buffer");
    if (mesh->device != ctx->device) return ctx_fail(ctx, LIAR_ERR_INVALID, "mesh lives on another device");
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    return launch_trace(ctx, mesh, d_rays, n_rays, d_hits, any_hit, nullptr, pick_stream(ctx, stream),
                        ctx->d_scratch + kCounterWord, ctx->d_scratch + kStatusWord);
}

extern "C" int liar_gpu_trace_counted_device(liar_gpu_ctx* ctx, const liar_gpu_mesh* mesh, const liar_ray* d_rays,
                                             size_t n_rays, liar_hit* d_hits, int any_hit,
                                             unsigned long long* d_counters, void* stream) {
    if (!ctx) return LIAR_ERR_INVALID;
    if (!mesh || !d_counters || (n_rays && (!d_rays || !d_hits)))
        return ctx_fail(ctx, LIAR_ERR_INVALID, "null mesh or buffer");
    if (mesh->device != ctx->device) return ctx_fail(ctx, LIAR_ERR_INVALID, "mesh lives on another device");
    if ((uintptr_t)d_counters & 7) return ctx_fail(ctx, LIAR_ERR_INVALID, "counters must be 8-byte aligned");
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    return launch_trace(ctx, mesh, d_rays, n_rays, d_hits, any_hit, reinterpret_cast<TraceCounters*>(d_counters),
                        pick_stream(ctx, stream), ctx->d_scratch + kCounterWord, ctx->d_scratch + kStatusWord);
}

extern "C" int liar_gpu_trace(liar_gpu_ctx* ctx, const liar_gpu_mesh* mesh, const liar_ray* rays, size_t n_rays,
                              liar_hit* hits, int any_hit) {
    if (!ctx) return LIAR_ERR_INVALID;
    if (!mesh || (n_rays && (!rays || !hits))) return ctx_fail(ctx, LIAR_ERR_INVALID, "null mesh or buffer");
    if (mesh->device != ctx->device) return ctx_fail(ctx, LIAR_ERR_INVALID, "mesh lives on another device");
    if (n_rays == 0) return LIAR_OK;
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    // Chunked pipeline: the copy in of chunk k+1 and the copy out of chunk k-1 overlap the
    // traversal of chunk k (PCIe, not the kernel, bounds this call). Up to kPipeSlots staging
    // slots, each with its own stream and work counter; chunks of 1M rays keep the unoverlapped
    // head (first copy in) and tail (last copy out) short.
    const size_t chunk = n_rays < (size_t)(1u << 20) ? n_rays : (size_t)(1u << 20);
    const size_t n_chunks = (n_rays + chunk - 1) / chunk;
    const int slots = n_chunks < (size_t)kPipeSlots ? (int)n_chunks : kPipeSlots;
    rc = ctx_grow(ctx, &ctx->d_rays, &ctx->cap_rays, (size_t)slots * chunk * sizeof(liar_ray), "ray staging buffer");
    if (rc) return rc;
    rc = ctx_grow(ctx, &ctx->d_hits, &ctx->cap_hits, (size_t)slots * chunk * sizeof(liar_hit), "hit staging buffer");
    if (rc) return rc;
    rc = ctx_ensure_pipeline(ctx);
    if (rc) return rc;
    liar_ray* dr = (liar_ray*)ctx->d_rays;
    liar_hit* dh = (liar_hit*)ctx->d_hits;
    // the pipeline streams wait for work already queued on the context stream
    cudaEventRecord(ctx->pipe_ev[kPipeSlots], ctx->stream);
    for (int s = 0; s < slots; ++s) cudaStreamWaitEvent(ctx->pipe[s], ctx->pipe_ev[kPipeSlots], 0);
    size_t k = 0;
    int slot = 0;
    for (size_t base = 0; base < n_rays; base += chunk, ++k, slot = (slot + 1) % slots) {
        const size_t m = (n_rays - base) < chunk ? (n_rays - base) : chunk;
        cudaStream_t st = ctx->pipe[slot];
        cudaError_t e = cudaMemcpyAsync(dr + (size_t)slot * chunk, rays + base, m * sizeof(liar_ray),
                                        cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "copy rays in");
        rc = launch_trace(ctx, mesh, dr + (size_t)slot * chunk, m, dh + (size_t)slot * chunk, any_hit, nullptr, st,
                          ctx->d_scratch + kCounterWord + 1 + slot, ctx->d_scratch + kStatusWord);
        if (rc) return rc;
        e = cudaMemcpyAsync(hits + base, dh + (size_t)slot * chunk, m * sizeof(liar_hit), cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "copy hits out");
    }
    // work queued on the context stream after this call is ordered after the whole trace
    for (int s = 0; s < slots; ++s) {
        cudaEventRecord(ctx->pipe_ev[s], ctx->pipe[s]);
        cudaStreamWaitEvent(ctx->stream, ctx->pipe_ev[s], 0);
    }
    for (int s = 0; s < slots; ++s) {
        rc = ctx_cuda(ctx, cudaStreamSynchronize(ctx->pipe[s]), "trace synchronize");
        if (rc) return rc;
    }
    return ctx_check_status(ctx);
}

extern "C" int liar_gpu_set_fault_test(liar_gpu_ctx* ctx, int mode) {
    if (!ctx) return LIAR_ERR_INVALID;
    if (mode != 0 && mode != LIAR_FAULT_TEST_GUIDE_WAIT) return ctx_fail(ctx, LIAR_ERR_INVALID, "fault test %d", mode);
    ctx->fault_test = mode;
    return LIAR_OK;
}

extern "C" int liar_gpu_set_cancel_flag(liar_gpu_ctx* ctx, const volatile int32_t* flag) {
    if (!ctx) return LIAR_ERR_INVALID;
    ctx->cancel_flag = flag;
    return LIAR_OK;
}

extern "C" int liar_gpu_set_trace_config(liar_gpu_ctx* ctx, const liar_trace_config* cfg) {
    if (!ctx || !cfg) return LIAR_ERR_INVALID;
    const int b = cfg->block_size, s = cfg->smem_stack;
    const bool ok = (b == 128 && (s == 8 || s == 16 || s == 24)) || (b == 256 && (s == 8 || s == 16));
    if (!ok) return ctx_fail(ctx, LIAR_ERR_INVALID, "unsupported trace config: block %d, shared stack %d", b, s);
    ctx->trace_cfg = *cfg;
    return LIAR_OK;
}

extern "C" int liar_gpu_get_trace_config(const liar_gpu_ctx* ctx, liar_trace_config* out) {
    if (!ctx || !out) return LIAR_ERR_INVALID;
    *out = ctx->trace_cfg;
    return LIAR_OK;
}
