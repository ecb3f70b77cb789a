// trace_noalloc.cu -- closest-hit / any-hit entry point that allocates no memory at all.
//
// Who needs it: code that must not call cudaMalloc while it traces. Examples are a host
// application that hands its whole device memory to its own pool allocator up front (a call to
// cudaMalloc then fails or steals memory the pool accounts for), a render loop that runs
// between frames with other streams busy (cudaMalloc / cudaFree can synchronise the device and
// stall them), and plugin hosts that give a plugin a fixed memory budget. Such a caller builds
// its meshes once during set-up (liar_gpu_mesh_build allocates) and then traces with
// liar_gpu_trace_device_noalloc on buffers it owns.
//
// The trace kernel needs a little scratch memory besides its inputs and outputs: the work
// counter its persistent warps pull rays from and the status word that reports a traversal
// stack overflow. Here that scratch is the file-scope array g_noalloc_scratch below, which is
// part of the library's device image: every GPU that loads the library holds its 256 bytes
// until the process exits. Host code cannot use the array's name as a device address (on the
// host the name denotes a host-side shadow), so the address is looked up once per device with
// cudaGetSymbolAddress, with that device current, on the first call made on that device.
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>

#include "../../include/liar_gpu.h"
#include "ctx.h"
#include "traverse.cuh"

using namespace liar_gpu;

namespace {

// word 0: work counter, word 1: status bits; the rest pads the array to its 256-byte alignment
constexpr int kNoAllocWords = 64;
__device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocWords];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
uint32_t* g_scratch_ptr[kMaxDevices] = {};
int g_num_sms[kMaxDevices] = {};
std::atomic<bool> g_ready[kMaxDevices] = {};

constexpr int kBlockNA = 128;
constexpr size_t kNoAllocMaxRays = (size_t)1 << 31;

// once per device, with that device current
int noalloc_setup(int device) {
    if (g_ready[device].load(std::memory_order_acquire)) return LIAR_OK;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (g_ready[device].load(std::memory_order_relaxed)) return LIAR_OK;
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || ptr == nullptr) {
        cudaGetLastError();
        return LIAR_ERR_CUDA;
    }
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess || sms <= 0) {
        cudaGetLastError();
        return LIAR_ERR_CUDA;
    }
    g_scratch_ptr[device] = static_cast<uint32_t*>(ptr);
    g_num_sms[device] = sms;
    g_ready[device].store(true, std::memory_order_release);
    return LIAR_OK;
}

template <bool ANY, int S>
int launch_noalloc(const QNode* nodes, const QTri* tris, const liar_ray* rays, uint32_t n, liar_hit* hits,
                   cudaStream_t st, uint32_t* scratch, int num_sms) {
    auto kern = trace_kernel<ANY, S, kBlockNA, false>;
    const size_t smem = (size_t)S * kBlockNA * 8;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return LIAR_ERR_CUDA;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBlockNA, smem) != cudaSuccess) {
        cudaGetLastError();
        return LIAR_ERR_CUDA;
    }
    if (per_sm <= 0) per_sm = 1;
    uint64_t blocks = (uint64_t)num_sms * per_sm;
    const uint64_t needed = ((uint64_t)n + kBlockNA - 1) / kBlockNA;
    if (blocks > needed) blocks = needed;
    // the array keeps whatever the previous call left: the counter and the status start at zero
    if (cudaMemsetAsync(scratch, 0, 2 * sizeof(uint32_t), st) != cudaSuccess) {
        cudaGetLastError();
        return LIAR_ERR_CUDA;
    }
    kern<<<(unsigned)blocks, kBlockNA, smem, st>>>(nodes, tris, rays, hits, n, scratch, scratch + 1, nullptr,
                                                   trace_batch(n, (uint32_t)blocks * (kBlockNA / 32)), nullptr);
    if (cudaGetLastError() != cudaSuccess) return LIAR_ERR_CUDA;
    return LIAR_OK;
}

}  // namespace

extern "C" int liar_gpu_trace_device_noalloc(const liar_gpu_mesh* mesh, const liar_ray* d_rays, size_t n_rays,
                                             liar_hit* d_hits, int any_hit, void* stream) {
    if (!mesh || (n_rays && (!d_rays || !d_hits))) return LIAR_ERR_INVALID;
    if (n_rays > kNoAllocMaxRays) return LIAR_ERR_INVALID;  // beyond what the 32-bit work counter can hand out
    if (((uintptr_t)d_rays & 15) || ((uintptr_t)d_hits & 7)) return LIAR_ERR_INVALID;
    if (n_rays == 0) return LIAR_OK;
    const int device = mesh_device(mesh);
    if (device < 0 || device >= kMaxDevices) return LIAR_ERR_INVALID;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) {
        cudaGetLastError();
        return LIAR_ERR_CUDA;
    }
    if (prev != device && cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return LIAR_ERR_CUDA;
    }
    int rc = noalloc_setup(device);
    const uint32_t need = mesh_stack_needed(mesh);
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t* scratch = g_scratch_ptr[device];
    const uint32_t n = (uint32_t)n_rays;
    if (rc == LIAR_OK) {
        if (need <= 24)
            rc = any_hit ? launch_noalloc<true, 24>(mesh_nodes(mesh), mesh_tris(mesh), d_rays, n, d_hits, st, scratch,
                                                    g_num_sms[device])
                         : launch_noalloc<false, 24>(mesh_nodes(mesh), mesh_tris(mesh), d_rays, n, d_hits, st, scratch,
                                                     g_num_sms[device]);
        else if (need <= 64)
            rc = any_hit ? launch_noalloc<true, 64>(mesh_nodes(mesh), mesh_tris(mesh), d_rays, n, d_hits, st, scratch,
                                                    g_num_sms[device])
                         : launch_noalloc<false, 64>(mesh_nodes(mesh), mesh_tris(mesh), d_rays, n, d_hits, st, scratch,
                                                     g_num_sms[device]);
        else
            rc = LIAR_ERR_STACK;
    }
    if (rc == LIAR_OK) {
        // wait, then report the kernel's status word (a stack overflow makes the result invalid)
        uint32_t status = 0;
        cudaError_t e = cudaStreamSynchronize(st);
        if (e == cudaSuccess) e = cudaMemcpy(&status, scratch + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            cudaGetLastError();
            rc = LIAR_ERR_CUDA;
        } else if (status & STATUS_STACK_OVERFLOW) {
            rc = LIAR_ERR_STACK;
        } else if (status) {
            rc = LIAR_ERR_CUDA;
        }
    }
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
    return rc;
}
