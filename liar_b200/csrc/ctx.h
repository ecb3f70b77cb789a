// ctx.h -- the opaque context behind liar_gpu_ctx, shared by the .cu files of the library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <functional>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/liar_gpu.h"
#include "qbvh.h"

namespace liar_gpu {

// Scratch words of a context (device memory, allocated once per context):
//   [kStatusWord]        device-side error bits, ORed by kernels, read and cleared by the host
//   [kCounterWord + k]   work counters of persistent kernels (k = 0 device calls, 1..kPipeSlots
//                        the host-buffer pipeline slots, above that other kernels)
constexpr int kScratchWords = 64;
constexpr int kStatusWord = 0;
constexpr int kCounterWord = 8;
constexpr uint32_t kStatusTimeout = 1u << 8;
constexpr int kPipeSlots = 3;  // staging slots of the host-buffer trace pipeline

}  // namespace liar_gpu

struct liar_gpu_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::string err;
    uint32_t* d_scratch = nullptr;
    // grow-only staging buffers of the host-buffer entry points
    void* d_rays = nullptr;
    size_t cap_rays = 0;
    void* d_hits = nullptr;
    size_t cap_hits = 0;
    cudaStream_t pipe[liar_gpu::kPipeSlots] = {};
    // pipe_ev[k]: end of slot k's work; pipe_ev[kPipeSlots]: start (work queued before the call)
    cudaEvent_t pipe_ev[liar_gpu::kPipeSlots + 1] = {};
    // launch shape of the trace kernels (liar_gpu_set_trace_config) and cached occupancy per kernel
    liar_trace_config trace_cfg{128, 16};
    std::unordered_map<const void*, int> occupancy;
    // the caller's cancel flag (liar_gpu_set_cancel_flag), read between waves and bounces
    const volatile int32_t* cancel_flag = nullptr;
    // LIAR_FAULT_TEST_* mode of liar_gpu_set_fault_test (0: off)
    int fault_test = 0;
    // resources of other subsystems (renderer, photon maps) register their release here
    std::vector<std::function<void()>> on_destroy;
    // per-subsystem state (work buffers of the renderer, photon maps), looked up by name
    std::vector<std::pair<std::string, void*>> extensions;

    void release_extensions() {
        for (auto it = on_destroy.rbegin(); it != on_destroy.rend(); ++it) (*it)();
        on_destroy.clear();
        for (int k = 0; k < liar_gpu::kPipeSlots; ++k)
            if (pipe[k]) cudaStreamDestroy(pipe[k]);
        for (int k = 0; k <= liar_gpu::kPipeSlots; ++k)
            if (pipe_ev[k]) cudaEventDestroy(pipe_ev[k]);
    }
};

namespace liar_gpu {

int ctx_fail(liar_gpu_ctx* ctx, int code, const char* fmt, ...);
int ctx_cuda(liar_gpu_ctx* ctx, cudaError_t e, const char* what);
int ctx_activate(liar_gpu_ctx* ctx);
int ctx_grow(liar_gpu_ctx* ctx, void** buf, size_t* cap, size_t bytes, const char* what);
int ctx_check_status(liar_gpu_ctx* ctx);

inline bool ctx_cancel_requested(const liar_gpu_ctx* ctx) { return ctx->cancel_flag && *ctx->cancel_flag != 0; }
// ends a cancelled render: waits for the work queued on st, then reports LIAR_ERR_CANCELLED
int ctx_cancelled(liar_gpu_ctx* ctx, cudaStream_t st);

inline int ctx_ensure_pipeline(liar_gpu_ctx* ctx) {
    for (int k = 0; k < kPipeSlots; ++k)
        if (!ctx->pipe[k]) {
            cudaError_t e = cudaStreamCreateWithFlags(&ctx->pipe[k], cudaStreamNonBlocking);
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "create pipeline stream");
        }
    for (int k = 0; k <= kPipeSlots; ++k)
        if (!ctx->pipe_ev[k]) {
            cudaError_t e = cudaEventCreateWithFlags(&ctx->pipe_ev[k], cudaEventDisableTiming);
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "create pipeline event");
        }
    return LIAR_OK;
}

// n_dev: when given, the ray count in device memory (at most n, which sizes the launch)
int trace_mesh_internal(liar_gpu_ctx* ctx, const liar_gpu_mesh* mesh, const liar_ray* d_rays, size_t n,
                        liar_hit* d_hits, int any_hit, cudaStream_t st, int counter_word,
                        const uint32_t* n_dev = nullptr);
const QNode* mesh_nodes(const liar_gpu_mesh* m);
const QTri* mesh_tris(const liar_gpu_mesh* m);
uint32_t mesh_stack_needed(const liar_gpu_mesh* m);
int mesh_device(const liar_gpu_mesh* m);
int mesh_build_with_spheres(liar_gpu_ctx* ctx, const float* vertices, size_t n_vertices, const uint32_t* triangles,
                            size_t n_triangles, const float* spheres, size_t n_spheres, const liar_build_opts* opts,
                            liar_gpu_mesh** out);

}  // namespace liar_gpu
