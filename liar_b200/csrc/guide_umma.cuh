// guide_umma.cuh -- the guide network's inference on the 5th-generation tensor cores (tcgen05).
//
// A CTA runs four independent 4-warp slots (inference, the training forward and backward), each
// evaluating 128 rows at a time (M = 128; thread r of the slot owns row r), so that one slot's SIMT
// work overlaps the others' tensor-core work.
//   * the weights live in shared memory as the B operands of every layer, bf16, K-major, in the
//     canonical no-swizzle layout: element (n, k) of a layer with K inputs at
//     (n / 8) * (K / 8) * 128 + (k / 8) * 128 + (n % 8) * 16 + (k % 8) * 2 bytes, i.e. 8x16-byte core
//     matrices with the K-adjacent ones 128 B apart (leading byte offset) and the 8-row groups
//     (K / 8) * 128 B apart (stride byte offset);
//   * the activations (A operands) use the same layout: 128 x 256 for the encodings (inference
//     streams them as four 128 x 64 K-chunks), 128 x 64 for the hidden layers;
//   * a slot's accumulator is 128 lanes x 64 f32 columns of tensor memory; its thread 0 issues each layer
//     as K / 16 tcgen05.mma (kind::f16, bf16 inputs, f32 accumulation) and commits them to an
//     mbarrier; every warp then reads its 32 lanes (tcgen05.ld 32x32b.x64), applies ReLU, and
//     writes the next layer's A operand back to shared memory.
// Every wait on the mbarrier is bounded; on a timeout the CTA records kStatusTimeout, frees its
// tensor memory and returns.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#include "guide_mlp.cuh"

namespace liar_gpu {
namespace guide {

constexpr int kTcRows = 128;

// B-operand images of the six layers (bytes from the start of the image)
__host__ __device__ constexpr uint32_t umma_w_offset(int l) {
    return l == 0 ? 0u : (l <= 5 ? 32768u + 8192u * (uint32_t)(l - 1) : 32768u + 4u * 8192u + 6144u);
}
constexpr uint32_t kUmmaWBytes = umma_w_offset(6);  // 71680
constexpr uint32_t kUmmaA0Bytes = (uint32_t)kTcRows * kEnc * 2;    // 65536
constexpr uint32_t kUmmaA1Bytes = (uint32_t)kTcRows * kWidth * 2;  // 16384

// Inference runs four slots per CTA (16 warps per SM). A slot's operand buffer holds two 128 x 64
// halves: layer 0's K = 256 is fed to the tensor core in four K-chunks of 64 encodings, chunk c in
// half c % 2 (the encodings of chunk c + 1 are written while chunk c's MMAs run), and the hidden
// activations use half 0. After the last layer the buffer stages the slot's 128 output rows (row
// pitch padded by 4 floats) for coalesced stores; a second area stages the 128 input rows.
constexpr int kEvSlots = 4;
constexpr int kEvThreads = 128 * kEvSlots;
constexpr uint32_t kEvTmemCols = 64 * kEvSlots;
constexpr uint32_t kEvHalf = (uint32_t)kTcRows * 64 * 2;  // 16384
constexpr uint32_t kEvBuf = 2 * kEvHalf;                   // 32768
constexpr uint32_t kEvIn = (uint32_t)kTcRows * 13 * 4;     // 6656: 128 training records of 13 floats
constexpr size_t kEvSmem = 1024 + kUmmaWBytes + (size_t)kEvSlots * (kEvBuf + kEvIn) + 128;

// byte offset of element (row, k) in a K-major no-swizzle operand with K columns
__host__ __device__ __forceinline__ uint32_t umma_offset(uint32_t row, uint32_t k, uint32_t K) {
    return (row >> 3) * (K >> 3) * 128u + (k >> 3) * 128u + (row & 7u) * 16u + (k & 7u) * 2u;
}

#ifdef __CUDACC__

// shared-memory matrix descriptor: start >> 4 [0,14), leading byte offset >> 4 [16,30),
// stride byte offset >> 4 [32,46), version 1 [46,48), no swizzle [61,64)
__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t smem_addr, uint32_t sbo_bytes) {
    return (uint64_t)((smem_addr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) |
           ((uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: f32 accumulator, bf16 A and B, both K-major, N, M = 128
__host__ __device__ constexpr uint32_t umma_idesc(uint32_t n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((uint32_t)(kTcRows >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint32_t mbar_addr) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar_addr)
                 : "memory");
}

// ---- TMA (tensor memory access) loads into this CTA's shared memory, completing on an mbarrier's
// transaction count; no cluster multicast (the source is always this GPU's own global memory)
__device__ __forceinline__ void mbar_init(uint32_t mbar_addr, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar_addr), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint32_t mbar_addr) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar_addr) : "memory");
}
// one arrival that also announces `bytes` of TMA transactions still to land on the barrier
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t mbar_addr, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar_addr), "r"(bytes) : "memory");
}
// box of a 2D / 3D tensor map at (x, y[, z]) -> shared memory; x * element size must be a multiple of
// 16 bytes (the innermost coordinate's alignment rule), rows past the tensor's extent read as zero
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const void* tmap, int x, int y, uint32_t mbar_addr) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(mbar_addr)
        : "memory");
}
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const void* tmap, int x, int y, int z, uint32_t mbar_addr) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(z), "r"(mbar_addr)
        : "memory");
}

// shared memory -> a 5D box of a tensor map in global memory (bulk async group of the issuing
// thread; rows past the tensor's extent are not written)
__device__ __forceinline__ void tma_store_5d(const void* tmap, int c0, int c1, int c2, int c3, int c4, uint32_t src) {
    asm volatile("cp.async.bulk.tensor.5d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4, %5}], [%6];" ::"l"(
                     reinterpret_cast<uint64_t>(tmap)),
                 "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(src)
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// shared memory -> a 2D box of a tensor map in global memory (bulk async group of the issuing thread)
__device__ __forceinline__ void tma_store_2d(const void* tmap, int x, int y, uint32_t src) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                     reinterpret_cast<uint64_t>(tmap)),
                 "r"(x), "r"(y), "r"(src)
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// the issuing thread's bulk stores have read their shared memory (it may be rewritten)
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// the issuing thread's bulk stores are complete
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// bounded wait for the mbarrier phase: true when it completed
__device__ __forceinline__ bool mbar_wait(uint32_t mbar_addr, uint32_t phase, uint32_t max_tries) {
    for (uint32_t i = 0; i < max_tries; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t"
            ".reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t"
            "}"
            : "=r"(done)
            : "r"(mbar_addr), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tmem_ld_x64(uint32_t taddr, float (&v)[64]) {
    uint32_t r[64];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x64.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,"
        "%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,"
        "%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
          "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]),
          "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]),
          "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
          "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 64; ++i) v[i] = __uint_as_float(r[i]);
}

template <int N>
__device__ __forceinline__ void tmem_ld_32x32b(uint32_t taddr, float* v);

// columns [c, c + 32) and [c, c + 8) of the warp's 32 lanes
template <>
__device__ __forceinline__ void tmem_ld_32x32b<32>(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

template <>
__device__ __forceinline__ void tmem_ld_32x32b<8>(uint32_t taddr, float* v) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Programmatic dependent launch: a kernel launched with programmatic stream serialization may start
// before the previous kernel of its stream has finished. grid_dependency_wait() blocks until that
// kernel has completed and its memory is visible (a no-op for a normally launched kernel); every
// read of its results, and every write it could still read, comes after. launch_dependents() lets
// the next such kernel start its own prologue; the kernels here call it only after their own wait,
// so a prologue never overlaps more than one kernel back.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// the encodings of row r into the 128 x 256 A operand: per input 12 sin/cos pairs = 3 chunks of
// 16 bytes (angle doubling as encode_row), then the raw inputs and zero padding
__device__ __forceinline__ void encode_row_umma(const float* x, unsigned char* a0, uint32_t r) {
    unsigned char* row = a0 + (r >> 3) * (kEnc / 8) * 128u + (r & 7u) * 16u;
#pragma unroll
    for (int d = 0; d < kIn; ++d) {
        float s0, c0, s1, c1;
        sincospi_enc(x[d], &s0, &c0);
        sincospi_enc(x[d] * 1.41421356237309515f, &s1, &c1);
        uint32_t w[12];
#pragma unroll
        for (int k = 0; k < kFreq / 2; ++k) {
            w[2 * k] = pack_bf16(s0, c0);
            w[2 * k + 1] = pack_bf16(s1, c1);
            const float ns0 = 2.0f * s0 * c0, nc0 = c0 * c0 - s0 * s0;
            const float ns1 = 2.0f * s1 * c1, nc1 = c1 * c1 - s1 * s1;
            s0 = ns0;
            c0 = nc0;
            s1 = ns1;
            c1 = nc1;
        }
#pragma unroll
        for (int c = 0; c < 3; ++c)
            *reinterpret_cast<uint4*>(row + (3 * d + c) * 128u) = make_uint4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]);
    }
    *reinterpret_cast<uint4*>(row + 27 * 128u) =
        make_uint4(pack_bf16(x[0], x[1]), pack_bf16(x[2], x[3]), pack_bf16(x[4], x[5]), pack_bf16(x[6], x[7]));
    *reinterpret_cast<uint4*>(row + 28 * 128u) = make_uint4(pack_bf16(x[8], 0.0f), 0u, 0u, 0u);
#pragma unroll
    for (int c = 29; c < kEnc / 8; ++c) *reinterpret_cast<uint4*>(row + c * 128u) = make_uint4(0u, 0u, 0u, 0u);
}

// The K-chunk c (encoding columns 64 c .. 64 c + 63) of row r, written into a 128 x 64 K-major
// operand buffer (the same values as encode_row_umma): the inputs whose 24 columns (3 core
// columns 3 d .. 3 d + 2) meet the chunk are encoded (an input that straddles two chunks is
// encoded in both), chunk 3 also holds the raw inputs and the zero padding.
// The same encodings for the K-chunks of 8 core columns as encode_chunk_umma, every input encoded
// once: input d fills core columns 3d .. 3d + 2, so inputs 2 (columns 6, 7 | 8) and 5 (15 | 16,
// 17) straddle a chunk boundary; their columns of the next chunk wait in carry (two columns of four
// words) and are written by the next call. Calls run for c = 0, 1, 2, 3 in order.
__device__ __forceinline__ void encode_chunk_carry(const float* x, unsigned char* a, uint32_t r, int c,
                                                   uint32_t (&carry)[8]) {
    unsigned char* row = a + (r >> 3) * 8u * 128u + (r & 7u) * 16u;
    const int lo = 8 * c, hi = 8 * c + 7;  // the chunk's core columns
    // the columns carried over from the previous chunk: 8 (c = 1), 16 and 17 (c = 2)
    if (c == 1) *reinterpret_cast<uint4*>(row) = make_uint4(carry[0], carry[1], carry[2], carry[3]);
    if (c == 2) {
        *reinterpret_cast<uint4*>(row) = make_uint4(carry[0], carry[1], carry[2], carry[3]);
        *reinterpret_cast<uint4*>(row + 128) = make_uint4(carry[4], carry[5], carry[6], carry[7]);
    }
#pragma unroll
    for (int d = 0; d < kIn; ++d) {
        if (3 * d < lo || 3 * d > hi) continue;  // an input belongs to the chunk of its first column
        uint32_t w[12];
        encode_input(x[d], w);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const int col = 3 * d + q;
            if (col <= hi) {
                *reinterpret_cast<uint4*>(row + (col - lo) * 128) = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
            } else {
                const int k = col - hi - 1;  // 0 or 1: its slot in the carry
                carry[4 * k] = w[4 * q];
                carry[4 * k + 1] = w[4 * q + 1];
                carry[4 * k + 2] = w[4 * q + 2];
                carry[4 * k + 3] = w[4 * q + 3];
            }
        }
    }
    if (c == 3) {
        *reinterpret_cast<uint4*>(row + (27 - lo) * 128) =
            make_uint4(pack_bf16(x[0], x[1]), pack_bf16(x[2], x[3]), pack_bf16(x[4], x[5]), pack_bf16(x[6], x[7]));
        *reinterpret_cast<uint4*>(row + (28 - lo) * 128) = make_uint4(pack_bf16(x[8], 0.0f), 0u, 0u, 0u);
#pragma unroll
        for (int col = 29; col < kEnc / 8; ++col) *reinterpret_cast<uint4*>(row + (col - lo) * 128) = make_uint4(0u, 0u, 0u, 0u);
    }
}

__device__ __forceinline__ void encode_chunk_umma(const float* x, unsigned char* a, uint32_t r, int c) {
    unsigned char* row = a + (r >> 3) * 8u * 128u + (r & 7u) * 16u;
    const int lo = 8 * c, hi = 8 * c + 7;  // the chunk's core columns
#pragma unroll
    for (int d = 0; d < kIn; ++d) {
        if (3 * d + 2 < lo || 3 * d > hi) continue;
        float s0, c0, s1, c1;
        sincospi_enc(x[d], &s0, &c0);
        sincospi_enc(x[d] * 1.41421356237309515f, &s1, &c1);
        uint32_t w[12];
#pragma unroll
        for (int k = 0; k < kFreq / 2; ++k) {
            w[2 * k] = pack_bf16(s0, c0);
            w[2 * k + 1] = pack_bf16(s1, c1);
            const float ns0 = 2.0f * s0 * c0, nc0 = c0 * c0 - s0 * s0;
            const float ns1 = 2.0f * s1 * c1, nc1 = c1 * c1 - s1 * s1;
            s0 = ns0;
            c0 = nc0;
            s1 = ns1;
            c1 = nc1;
        }
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const int col = 3 * d + q;
            if (col >= lo && col <= hi)
                *reinterpret_cast<uint4*>(row + (col - lo) * 128) = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
        }
    }
    if (c == 3) {
        *reinterpret_cast<uint4*>(row + (27 - lo) * 128) =
            make_uint4(pack_bf16(x[0], x[1]), pack_bf16(x[2], x[3]), pack_bf16(x[4], x[5]), pack_bf16(x[6], x[7]));
        *reinterpret_cast<uint4*>(row + (28 - lo) * 128) = make_uint4(pack_bf16(x[8], 0.0f), 0u, 0u, 0u);
#pragma unroll
        for (int col = 29; col < kEnc / 8; ++col) *reinterpret_cast<uint4*>(row + (col - lo) * 128) = make_uint4(0u, 0u, 0u, 0u);
    }
}

#endif  // __CUDACC__

}  // namespace guide
}  // namespace liar_gpu
