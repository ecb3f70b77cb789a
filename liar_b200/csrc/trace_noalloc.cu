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
constexpr int kBlockNA = 128;
// the context path's default launch shape: 16 stack entries per lane in shared memory, the rest
// (up to 64) in local memory; a program that has traced through a context has this kernel loaded
constexpr int kStackNA = 16;
constexpr size_t kNoAllocMaxRays = (size_t)1 << 31;

struct NoAllocDevice {
    uint32_t* scratch = nullptr;  // device address of g_noalloc_scratch on this device
    unsigned blocks[2] = {};      // persistent grid of the closest-hit [0] and any-hit [1] kernel
};
std::mutex g_setup_mutex;
NoAllocDevice g_dev[kMaxDevices];
std::atomic<bool> g_ready[kMaxDevices] = {};

template <bool ANY>
int resident_blocks(int sms, unsigned* out) {
    auto kern = trace_kernel<ANY, kStackNA, kBlockNA, false>;
    const size_t smem = (size_t)kStackNA * kBlockNA * 8;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBlockNA, smem) != cudaSuccess) {
        cudaGetLastError();
        return LIAR_ERR_CUDA;
    }
    *out = (unsigned)sms * (unsigned)(per_sm > 0 ? per_sm : 1);
    return LIAR_OK;
}

// once per device, with that device current: the scratch array's device address and the grid
// sizes, so that later calls make no driver queries
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
    NoAllocDevice d;
    d.scratch = static_cast<uint32_t*>(ptr);
    int rc = resident_blocks<false>(sms, &d.blocks[0]);
    if (rc == LIAR_OK) rc = resident_blocks<true>(sms, &d.blocks[1]);
    if (rc != LIAR_OK) return rc;
    g_dev[device] = d;
    g_ready[device].store(true, std::memory_order_release);
    return LIAR_OK;
}

template <bool ANY>
int launch_noalloc(const QNode* nodes, const QTri* tris, const liar_ray* rays, uint32_t n, liar_hit* hits,
                   cudaStream_t st, const NoAllocDevice& d) {
    const size_t smem = (size_t)kStackNA * kBlockNA * 8;
    uint64_t blocks = d.blocks[ANY ? 1 : 0];
    const uint64_t needed = ((uint64_t)n + kBlockNA - 1) / kBlockNA;
    if (blocks > needed) blocks = needed;
    // the array keeps whatever the previous call left: the counter and the status start at zero
    if (cudaMemsetAsync(d.scratch, 0, 2 * sizeof(uint32_t), st) != cudaSuccess) {
        cudaGetLastError();
        return LIAR_ERR_CUDA;
    }
    trace_kernel<ANY, kStackNA, kBlockNA, false><<<(unsigned)blocks, kBlockNA, smem, st>>>(
        nodes, tris, rays, hits, n, d.scratch, d.scratch + 1, nullptr,
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
    const uint32_t n = (uint32_t)n_rays;
    if (rc == LIAR_OK) {
        if (need > (uint32_t)kTraceStackTotal)
            rc = LIAR_ERR_STACK;
        else
            rc = any_hit ? launch_noalloc<true>(mesh_nodes(mesh), mesh_tris(mesh), d_rays, n, d_hits, st, g_dev[device])
                         : launch_noalloc<false>(mesh_nodes(mesh), mesh_tris(mesh), d_rays, n, d_hits, st, g_dev[device]);
    }
    if (rc == LIAR_OK) {
        // read the kernel's status word on the caller's stream, then wait for that stream only
        // (a stack overflow makes the result invalid)
        uint32_t status = 0;
        cudaError_t e = cudaMemcpyAsync(&status, g_dev[device].scratch + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
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
