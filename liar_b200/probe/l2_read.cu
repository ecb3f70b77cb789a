// l2_read.cu -- the L2 read-bandwidth probe of the benchmark (not part of the library's C ABI).
//
// The trace kernel's traffic is mostly tree nodes and triangles served from L2, so its roofline
// needs an L2 bandwidth beside the HBM copy bandwidth. This kernel reads a buffer that fits in L2
// (the caller sizes it) again and again with 16-byte loads, every SM taking a grid-stride share,
// and folds what it reads into one word per thread so the loads cannot be dropped. Bytes read over
// the kernel's duration is the L2 read bandwidth a streaming reader can reach.
#include <cuda_runtime.h>
#include <stdint.h>

namespace {

__global__ void __launch_bounds__(512) k_l2_read(const uint4* __restrict__ buf, uint64_t n_vec, int passes,
                                                 uint32_t* __restrict__ sink) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint32_t acc = 0;
    for (int p = 0; p < passes; ++p) {
#pragma unroll 4
        for (uint64_t i = tid; i < n_vec; i += stride) {
            const uint4 v = __ldcg(buf + i);  // cached in L2 only, as the trace kernel's node loads
            acc ^= v.x ^ v.y ^ v.z ^ v.w;
        }
    }
    sink[tid] = acc;
}

}  // namespace

// Reads n_vec 16-byte words of buf `passes` times on `stream`; sink holds one word per thread of
// the grid (blocks x 512). Returns 0, or the CUDA error code of the launch.
extern "C" int liar_probe_l2_read(const void* buf, uint64_t n_vec, int passes, int blocks, uint32_t* sink,
                                  void* stream) {
    if (!buf || !sink || n_vec == 0 || passes <= 0 || blocks <= 0) return (int)cudaErrorInvalidValue;
    k_l2_read<<<(unsigned)blocks, 512, 0, (cudaStream_t)stream>>>(static_cast<const uint4*>(buf), n_vec, passes, sink);
    return (int)cudaGetLastError();
}
