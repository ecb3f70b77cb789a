// guide.cu -- the path-guiding network: inference, online training (Adam), and its C ABI
// (no reference counterpart; the reference's AdjointPhotonTracer samples BSDF and lights only,
// src/liar/tracers/adjoint_photon_tracer.cpp:212-292).
//
// Training minimises the KL divergence from the normalised integrand to the guide
// (neural importance sampling, Mueller et al. 2019): for records (x, w, F/p) the loss is
//   L = -(1/B) sum_i min((F_i/p_i) / mean(F/p), 20) * log q(w_i | x_i),
// q = sum_l pi_l vMF(w; mu_l, kappa_l), pi = softmax(logits), mu = m / |m|, kappa = e^{clamp(s)}.
// One step: forward (stores the bf16 activations and the output gradient, fused) -> backward
// (stores the bf16 layer deltas) -> weight gradients as split-K GEMMs over the records ->
// Adam on the f32 master weights -> repack the bf16 fragments.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "../../include/liar_gpu.h"
#include "ctx.h"
#include "guide_mlp.cuh"
#include "guide_umma.cuh"
#include "sampler.h"

using namespace liar_gpu;
using namespace liar_gpu::guide;

struct liar_gpu_guide {
    int device = -1;
    liar_guide_config cfg{};
    float* params = nullptr;   // f32 master weights
    float* grads = nullptr;
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    uint32_t* step = nullptr;  // Adam step count (device)
    uint2* frag_fwd = nullptr;
    uint2* frag_bwd = nullptr;
    unsigned char* umma_w = nullptr;  // B-operand images of the six layers for the tcgen05 inference
    // training scratch, sized for cap records
    size_t cap = 0;
    __nv_bfloat16* enc = nullptr;    // h_0 (the encodings): [cap][256]
    __nv_bfloat16* act = nullptr;    // h_1..h_5: [5][cap][64]
    __nv_bfloat16* delta = nullptr;  // delta_1..delta_5: [5][cap][64]
    __nv_bfloat16* gout = nullptr;   // [cap][48]
    float* scalars = nullptr;        // [0] weight sum [1] loss sum
    std::vector<void*> buffers;
    unsigned long long steps_done = 0;
    unsigned long long records = 0, guided = 0, passes = 0;
};

namespace liar_gpu {
namespace guide {
// used by the guided renderer (guided.cu)
const uint2* guide_frag_fwd(const liar_gpu_guide* g) { return g->frag_fwd; }
const liar_guide_config& guide_config(const liar_gpu_guide* g) { return g->cfg; }
int guide_device(const liar_gpu_guide* g) { return g->device; }
unsigned long long guide_steps(const liar_gpu_guide* g) { return g->steps_done; }
void guide_count(liar_gpu_guide* g, unsigned long long records, unsigned long long guided, unsigned long long passes) {
    g->records += records;
    g->guided += guided;
    g->passes += passes;
}
int guide_train(liar_gpu_ctx* ctx, liar_gpu_guide* g, const float* d_records, const uint32_t* d_count, size_t n_max,
                int apply, float* d_grad_out, float* d_loss_out, cudaStream_t st);
}  // namespace guide
}  // namespace liar_gpu

namespace {

constexpr int kThreads = 128;  // 4 warps
constexpr int kRecordFloats = 13;
// normalised record weights are clipped here: radiance estimates are heavy-tailed and a handful of
// records would otherwise set the whole gradient (the renderer stays unbiased whatever the guide)
constexpr float kWeightClip = 20.0f;
constexpr int kFwdWarps = 8;  // forward kernels: 8 warps share one copy of the weights
constexpr int kFwdThreads = 32 * kFwdWarps;
// per warp: the encodings of its 32 rows; the raw outputs reuse the same bytes afterwards
static_assert((size_t)32 * kOutStride * sizeof(float) <= kEncWarpBytes, "output scratch fits the encodings");
constexpr size_t kEvalSmem = kFwdBytes + kFwdWarps * kEncWarpBytes;

__device__ __forceinline__ void normalise_input(const float* raw, const float* lo, const float* inv_ext, float* x) {
    for (int c = 0; c < 3; ++c) x[c] = (raw[c] - lo[c]) * inv_ext[c];
    for (int c = 3; c < kIn; ++c) x[c] = raw[c];
}

struct Box {
    float lo[3], inv_ext[3];
};

Box make_box(const liar_guide_config& c) {
    Box b;
    for (int k = 0; k < 3; ++k) {
        b.lo[k] = c.bounds_lo[k];
        const float e = c.bounds_hi[k] - c.bounds_lo[k];
        b.inv_ext[k] = e > 0 ? 1.0f / e : 0.0f;
    }
    return b;
}

// ---- fragments

__global__ void k_pack(const float* __restrict__ P, uint2* __restrict__ fwd, uint2* __restrict__ bwd,
                       uint32_t* step, int bump) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = i & 31, g = lane >> 2, t = lane & 3;
    const int tile = i >> 5;
    if (i == 0 && bump) *step += 1;
    auto bf = [](float v) { return __float2bfloat16_rn(v); };
    auto pk = [&](float a, float b) {
        __nv_bfloat162 v;
        v.x = bf(a);
        v.y = bf(b);
        return *reinterpret_cast<uint32_t*>(&v);
    };
    if (tile < kFwdTiles) {
        int l = 0;
        while (l < 5 && tile >= fwd_tile_offset(l + 1)) ++l;
        const int loc = tile - fwd_tile_offset(l), N = layer_n(l);
        const int kk = loc / (N / 8), nt = loc % (N / 8);
        const int k0 = 16 * kk + 2 * t, n = 8 * nt + g;
        const float* W = P + param_offset(l);
        fwd[i] = make_uint2(pk(W[k0 * N + n], W[(k0 + 1) * N + n]), pk(W[(k0 + 8) * N + n], W[(k0 + 9) * N + n]));
    } else if (tile < kFwdTiles + kBwdTiles) {
        const int bt = tile - kFwdTiles;
        int l = 1;
        while (l < 5 && bt >= bwd_tile_offset(l + 1)) ++l;
        const int loc = bt - bwd_tile_offset(l), N = layer_n(l);
        const int kk = loc / 8, nt = loc % 8;
        const int k0 = 16 * kk + 2 * t, n = 8 * nt + g;  // k over the out features, n over the in features
        const float* W = P + param_offset(l);
        bwd[(size_t)bt * 32 + lane] =
            make_uint2(pk(W[n * N + k0], W[n * N + k0 + 1]), pk(W[n * N + k0 + 8], W[n * N + k0 + 9]));
    }
}

// the tcgen05 B operands: layer l's element (n, k) = W_l[k][n] at umma_offset(n, k, K_l)
__global__ void k_pack_umma(const float* __restrict__ P, unsigned char* __restrict__ img) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;  // one parameter (k, n) per thread
    if (i >= kParams) return;
    int l = 0;
    while (l < 5 && i >= param_offset(l + 1)) ++l;
    const int loc = i - param_offset(l), N = layer_n(l), K = layer_k(l);
    const int k = loc / N, n = loc % N;
    *reinterpret_cast<__nv_bfloat16*>(img + umma_w_offset(l) + umma_offset((uint32_t)n, (uint32_t)k, (uint32_t)K)) =
        __float2bfloat16_rn(P[i]);
}

int launch_pack(liar_gpu_guide* G, cudaStream_t st, int bump) {
    const int total = (kFwdTiles + kBwdTiles) * 32;
    k_pack<<<(total + 255) / 256, 256, 0, st>>>(G->params, G->frag_fwd, G->frag_bwd, G->step, bump);
    k_pack_umma<<<(kParams + 255) / 256, 256, 0, st>>>(G->params, G->umma_w);
    return cudaGetLastError() == cudaSuccess ? LIAR_OK : LIAR_ERR_CUDA;
}

__device__ __forceinline__ void load_frags(uint2* dst, const uint2* __restrict__ src, size_t bytes) {
    const uint4* s = reinterpret_cast<const uint4*>(src);
    uint4* d = reinterpret_cast<uint4*>(dst);
    for (size_t i = threadIdx.x; i < bytes / 16; i += blockDim.x) d[i] = s[i];
    __syncthreads();
}

// ---- inference on tcgen05: two slots of 128 rows per CTA (guide_umma.cuh)
// Every mbarrier wait is bounded by max_tries polls. A wait that runs out records the timeout,
// waits once more (bounded again) for the commit it was waiting for, so that no MMA still writes
// the accumulator, and the CTA frees its TMEM and leaves. issue_mma = 0 is the timeout test: no
// MMA and no commit are issued, so the first wait runs out with nothing in flight.
__global__ void __launch_bounds__(kTcThreads, 1) k_eval_tc(const unsigned char* __restrict__ w_img,
                                                           const float* __restrict__ in, size_t n, Box box,
                                                           float* __restrict__ mix, int stride,
                                                           uint32_t* __restrict__ status, uint32_t max_tries,
                                                           int issue_mma) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char* sw = smem;
    uint64_t* mbar_all = reinterpret_cast<uint64_t*>(sw + kUmmaWBytes + (size_t)kTcSlots * kUmmaA0Bytes);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar_all + kTcSlots);
    volatile uint32_t* failed = tmem_slot + 1;  // one flag per slot
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    const uint32_t slot = tid >> 7, r = tid & 127u;  // this thread's slot and row within the slot's tile
    unsigned char* buf = sw + kUmmaWBytes + slot * kUmmaA0Bytes;
    {
        const uint4* s = reinterpret_cast<const uint4*>(w_img);
        uint4* d = reinterpret_cast<uint4*>(sw);
        for (uint32_t i = tid; i < kUmmaWBytes / 16; i += kTcThreads) d[i] = s[i];
    }
    if (tid == 0) {
        for (int k = 0; k < kTcSlots; ++k)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((uint32_t)__cvta_generic_to_shared(mbar_all + k)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        failed[0] = failed[1] = 0u;
    }
    if (warp == 0) {
        const uint32_t sa = (uint32_t)__cvta_generic_to_shared(tmem_slot);
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sa), "r"(kTcTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot + 64u * slot;                 // the slot's accumulator columns
    const uint32_t taddr = tmem + ((32u * (warp & 3u)) << 16);     // the warp's lane quarter
    const uint32_t mbar_addr = (uint32_t)__cvta_generic_to_shared(mbar_all + slot);
    const uint32_t sw_addr = (uint32_t)__cvta_generic_to_shared(sw);
    const uint32_t buf_addr = (uint32_t)__cvta_generic_to_shared(buf);
    auto slot_sync = [&]() { asm volatile("bar.sync %0, 128;" ::"r"(1u + slot) : "memory"); };
    uint32_t phase = 0;
    const size_t n_tiles = (n + kTcRows - 1) / kTcRows;
    for (size_t tile = (size_t)blockIdx.x * kTcSlots + slot; tile < n_tiles; tile += (size_t)gridDim.x * kTcSlots) {
        const size_t row = tile * kTcRows + r;
        float x[kIn];
        if (row < n) normalise_input(in + row * kIn, box.lo, box.inv_ext, x);
        else
            for (int c = 0; c < kIn; ++c) x[c] = 0.0f;
        encode_row_umma(x, buf, r);
        float v[64];
        bool ok = true;
        for (int l = 0; l < kLayers; ++l) {
            // the layer's A operand is in shared memory and the slot's last accumulator reads are
            // done: hand the operand to the tensor core
            fence_async_smem();
            tc_fence_before();
            slot_sync();
            tc_fence_after();
            if (r == 0 && issue_mma) {
                const uint32_t K = (uint32_t)layer_k(l), N = (uint32_t)layer_n(l);
                const uint32_t b_base = sw_addr + umma_w_offset(l);
                const uint32_t idesc = umma_idesc(N);
                for (uint32_t j = 0; j < K / 16; ++j)
                    umma_bf16(tmem, umma_smem_desc(buf_addr + 256u * j, (K / 8) * 128u),
                              umma_smem_desc(b_base + 256u * j, (K / 8) * 128u), idesc, j > 0 ? 1u : 0u);
                umma_commit(mbar_addr);
            }
            if (!mbar_wait(mbar_addr, phase, max_tries)) failed[slot] = 1u;
            slot_sync();  // the slot agrees on completion before anyone reads the accumulator
            if (failed[slot]) {
                // drain: the commit this slot gave up on, if any, before the TMEM is freed
                if (issue_mma) mbar_wait(mbar_addr, phase, max_tries);
                ok = false;
                break;
            }
            phase ^= 1u;
            tc_fence_after();
            tmem_ld_x64(taddr, v);
            if (l < kLayers - 1) {
                // ReLU, bf16, the next layer's A operand (row r, 8 chunks of 8 columns) in the slot's
                // buffer, whose encodings the finished layer-0 MMA no longer needs
                unsigned char* dst = buf + (r >> 3) * (kWidth / 8) * 128u + (r & 7u) * 16u;
#pragma unroll
                for (int c = 0; c < kWidth / 8; ++c) {
                    const float* q = v + 8 * c;
                    *reinterpret_cast<uint4*>(dst + c * 128u) =
                        make_uint4(pack_bf16(fmaxf(q[0], 0.0f), fmaxf(q[1], 0.0f)), pack_bf16(fmaxf(q[2], 0.0f), fmaxf(q[3], 0.0f)),
                                   pack_bf16(fmaxf(q[4], 0.0f), fmaxf(q[5], 0.0f)), pack_bf16(fmaxf(q[6], 0.0f), fmaxf(q[7], 0.0f)));
                }
            }
        }
        if (!ok) break;
        if (row < n) {
            Lobe lobes[kLobes];
            float w[kLobes];
            mixture_from_raw(v, lobes, w);
            float4* dst = reinterpret_cast<float4*>(mix + row * (size_t)stride);
            for (int l = 0; l < kLobes; ++l) dst[l] = make_float4(lobes[l].mx, lobes[l].my, lobes[l].mz, lobes[l].kappa);
            dst[8] = make_float4(w[0], w[1], w[2], w[3]);
            dst[9] = make_float4(w[4], w[5], w[6], w[7]);
            if (stride == kMixRender) {
                float a[kLobes];
                for (int l = 0; l < kLobes; ++l) a[l] = w[l] * vmf_norm(lobes[l].kappa);
                dst[10] = make_float4(a[0], a[1], a[2], a[3]);
                dst[11] = make_float4(a[4], a[5], a[6], a[7]);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*tmem_slot), "r"(kTcTmemCols));
    if (tid == 0 && (failed[0] | failed[1])) atomicOr(status, kStatusTimeout);
}

// ---- training

__global__ void k_weight_sum(const float* __restrict__ rec, const uint32_t* __restrict__ n_dev, size_t n_max,
                             float* scalars) {
    const size_t n = n_dev ? min((size_t)*n_dev, n_max) : n_max;
    float s = 0.0f;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float w = rec[i * kRecordFloats + 12];
        if (w > 0.0f && isfinite(w)) s += w;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0 && s != 0.0f) atomicAdd(scalars, s);
}

// the loss gradient of one record with respect to the 40 raw outputs (scaled by `scale`)
__device__ float record_gradient(const float* o, float wx, float wy, float wz, float weight, float scale, float* d) {
    Lobe L[kLobes];
    float pi[kLobes], la[kLobes], cs[kLobes];
    mixture_from_raw(o, L, pi);
    float mx = -3.0e38f;
    for (int l = 0; l < kLobes; ++l) {
        cs[l] = L[l].mx * wx + L[l].my * wy + L[l].mz * wz;
        la[l] = logf(pi[l]) + vmf_log_pdf(L[l].kappa, cs[l]);
        mx = fmaxf(mx, la[l]);
    }
    float s = 0.0f;
    for (int l = 0; l < kLobes; ++l) s += expf(la[l] - mx);
    const float lq = mx + logf(s);
    const float ws = weight * scale;
    for (int l = 0; l < kLobes; ++l) {
        const float r = expf(la[l] - lq);
        const float k = L[l].kappa;
        const float c = -ws * r;
        d[5 * l + 4] = -ws * (r - pi[l]);
        const float sk = o[5 * l + 3];
        d[5 * l + 3] = (sk > kLogKappaMin && sk < kLogKappaMax) ? c * k * (1.0f / k - 2.0f / expm1f(2.0f * k) + cs[l] - 1.0f)
                                                                 : 0.0f;
        // d mu / d m = (I - mu mu^T) / |m|
        const float nm = sqrtf(o[5 * l] * o[5 * l] + o[5 * l + 1] * o[5 * l + 1] + o[5 * l + 2] * o[5 * l + 2]);
        const float f = c * k / fmaxf(nm, kMeanNormMin);
        d[5 * l + 0] = f * (wx - cs[l] * L[l].mx);
        d[5 * l + 1] = f * (wy - cs[l] * L[l].my);
        d[5 * l + 2] = f * (wz - cs[l] * L[l].mz);
    }
    return -weight * lq;
}

// forward over a batch of records with the activations stored, then the output gradient
__global__ void __launch_bounds__(kFwdThreads) k_train_forward(const uint2* __restrict__ frag, const float* __restrict__ rec,
                                                               const uint32_t* __restrict__ n_dev, size_t n_max, Box box,
                                                               const float* __restrict__ scalars_in,
                                                               __nv_bfloat16* __restrict__ enc_out,
                                                               __nv_bfloat16* __restrict__ act,
                                                               __nv_bfloat16* __restrict__ gout, float* __restrict__ loss) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint2* wf = reinterpret_cast<uint2*>(smem);
    load_frags(wf, frag, kFwdBytes);
    const size_t n = n_dev ? min((size_t)*n_dev, n_max) : n_max;
    const float wsum = scalars_in[0];
    const float inv_mean = (wsum > 0.0f && n > 0) ? (float)n / wsum : 0.0f;
    const float inv_b = n > 0 ? 1.0f / (float)n : 0.0f;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __nv_bfloat16* enc = reinterpret_cast<__nv_bfloat16*>(smem + kFwdBytes + warp * kEncWarpBytes);
    float* os = reinterpret_cast<float*>(enc);
    const size_t n_tiles = (n + 31) / 32;
    float lsum = 0.0f;
    for (size_t tile = (size_t)blockIdx.x * kFwdWarps + warp; tile < n_tiles; tile += (size_t)gridDim.x * kFwdWarps) {
        const size_t row = tile * 32 + lane;
        float x[kIn];
        float wx = 0, wy = 0, wz = 1, weight = 0;
        if (row < n) {
            const float* r = rec + row * kRecordFloats;
            normalise_input(r, box.lo, box.inv_ext, x);
            wx = r[9];
            wy = r[10];
            wz = r[11];
            weight = r[12];
            if (!(weight > 0.0f) || !isfinite(weight)) weight = 0.0f;
        } else {
            for (int c = 0; c < kIn; ++c) x[c] = 0.0f;
        }
        encode_row(x, enc + lane * kEncLd);
        __syncwarp();
        const uint32_t valid = (uint32_t)min((size_t)32, n - tile * 32);
        // h_0 for the weight gradient of W0: the warp writes its rows, 512 contiguous bytes each
        for (uint32_t r = 0; r < valid; ++r)
            reinterpret_cast<uint4*>(enc_out + (tile * 32 + r) * kEnc)[lane] =
                reinterpret_cast<const uint4*>(enc + r * kEncLd)[lane];
        float out[2][6][4];
        mlp_forward_warp(enc, wf, out, ActStore{act, n_max * kWidth, (uint32_t)(tile * 32), valid});
        __syncwarp();
        scatter_out(out, os);
        __syncwarp();
        if (row < n) {
            float d[kOut];
            for (int c = kOutUsed; c < kOut; ++c) d[c] = 0.0f;
            const float wn = fminf(weight * inv_mean, kWeightClip);
            lsum += record_gradient(os + lane * kOutStride, wx, wy, wz, wn, inv_b, d);
            uint32_t* dst = reinterpret_cast<uint32_t*>(gout + row * kOut);
            for (int c = 0; c < kOut / 2; ++c) dst[c] = pack_bf16(d[2 * c], d[2 * c + 1]);
        }
        __syncwarp();
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, o);
    if (lane == 0 && lsum != 0.0f) atomicAdd(loss, lsum * inv_b);
}

// backward: delta_5 = (g_out W5^T) * [h_5 > 0], ..., delta_1 = (delta_2 W1^T) * [h_1 > 0]
__global__ void __launch_bounds__(kThreads) k_train_backward(const uint2* __restrict__ frag_bwd,
                                                             const uint32_t* __restrict__ n_dev, size_t n_max,
                                                             const __nv_bfloat16* __restrict__ act,
                                                             const __nv_bfloat16* __restrict__ gout,
                                                             __nv_bfloat16* __restrict__ delta) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint2* wb = reinterpret_cast<uint2*>(smem);
    load_frags(wb, frag_bwd, kBwdBytes);
    const size_t n = n_dev ? min((size_t)*n_dev, n_max) : n_max;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const size_t n_tiles = (n + 31) / 32;
    for (size_t tile = (size_t)blockIdx.x * 4 + warp; tile < n_tiles; tile += (size_t)gridDim.x * 4) {
        const size_t r0 = tile * 32;
        auto ld32 = [&](const __nv_bfloat16* base, size_t ld, size_t row, int col) -> uint32_t {
            return row < n ? *reinterpret_cast<const uint32_t*>(base + row * ld + col) : 0u;
        };
        // A fragments of g_out (3 k tiles of 16 over the 48 outputs)
        uint32_t a[2][4][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int kk = 0; kk < 3; ++kk) {
                const size_t ra = r0 + 16 * mt + g;
                a[mt][kk][0] = ld32(gout, kOut, ra, 16 * kk + 2 * t);
                a[mt][kk][1] = ld32(gout, kOut, ra + 8, 16 * kk + 2 * t);
                a[mt][kk][2] = ld32(gout, kOut, ra, 16 * kk + 8 + 2 * t);
                a[mt][kk][3] = ld32(gout, kOut, ra + 8, 16 * kk + 8 + 2 * t);
            }
#pragma unroll 1
        for (int l = 5; l >= 1; --l) {
            const int n_kk = layer_n(l) / 16;  // 3 for W5, 4 otherwise
            float acc[2][8][4];
#pragma unroll
            for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                for (int nt = 0; nt < 8; ++nt)
#pragma unroll
                    for (int r = 0; r < 4; ++r) acc[mt][nt][r] = 0.0f;
            const uint2* wl = wb + (size_t)bwd_tile_offset(l) * 32 + lane;
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                if (kk < n_kk) {
#pragma unroll
                    for (int nt = 0; nt < 8; ++nt) {
                        const uint2 b = wl[(kk * 8 + nt) * 32];
                        mma_bf16(acc[0][nt], a[0][kk], b);
                        mma_bf16(acc[1][nt], a[1][kk], b);
                    }
                }
            }
            // mask by h_l > 0, store delta_l, regroup as A fragments for the next layer down
            const __nv_bfloat16* h = act + (size_t)(l - 1) * n_max * kWidth;
            __nv_bfloat16* dl = delta + (size_t)(l - 1) * n_max * kWidth;
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                const size_t ra = r0 + 16 * mt + g, rb = ra + 8;
#pragma unroll
                for (int nt = 0; nt < 8; ++nt) {
                    const int c = 8 * nt + 2 * t;
                    const uint32_t ha = ld32(h, kWidth, ra, c), hb = ld32(h, kWidth, rb, c);
                    float* v = acc[mt][nt];
                    if (!(bf16_lo(ha) > 0.0f)) v[0] = 0.0f;
                    if (!(bf16_hi(ha) > 0.0f)) v[1] = 0.0f;
                    if (!(bf16_lo(hb) > 0.0f)) v[2] = 0.0f;
                    if (!(bf16_hi(hb) > 0.0f)) v[3] = 0.0f;
                    const uint32_t pa = pack_bf16(v[0], v[1]), pb = pack_bf16(v[2], v[3]);
                    if (ra < n) *reinterpret_cast<uint32_t*>(dl + ra * kWidth + c) = pa;
                    if (rb < n) *reinterpret_cast<uint32_t*>(dl + rb * kWidth + c) = pb;
                    const int kk = nt >> 1;
                    if ((nt & 1) == 0) {
                        a[mt][kk][0] = pa;
                        a[mt][kk][1] = pb;
                    } else {
                        a[mt][kk][2] = pa;
                        a[mt][kk][3] = pb;
                    }
                }
            }
        }
    }
}

// weight gradients: dW_l = H_l^T D_l summed over the records, split over record chunks.
// job 0..3: W0 rows [64 j, 64 j + 64) (H = the encoding, D = delta_1); job 4..7: W1..W4
// (H = h_l, D = delta_{l+1}); job 8: W5 (H = h_5, D = g_out, 48 wide).
constexpr int kDwChunk = 2048;
constexpr int kDwStage = 64;
constexpr int kDwLd = 72;  // padded bf16 row stride of the staged tiles

__global__ void __launch_bounds__(kThreads) k_train_dw(const uint32_t* __restrict__ n_dev, size_t n_max,
                                                       const __nv_bfloat16* __restrict__ enc,
                                                       const __nv_bfloat16* __restrict__ act,
                                                       const __nv_bfloat16* __restrict__ delta,
                                                       const __nv_bfloat16* __restrict__ gout, float* __restrict__ grads) {
    __shared__ __align__(16) uint16_t Hs[kDwStage * kDwLd];
    __shared__ __align__(16) uint16_t Ds[kDwStage * kDwLd];
    const size_t n = n_dev ? min((size_t)*n_dev, n_max) : n_max;
    const int job = blockIdx.y;
    const size_t c0 = (size_t)blockIdx.x * kDwChunk;
    if (c0 >= n) return;
    const size_t c1 = min(n, c0 + kDwChunk);
    const int layer = job < 4 ? 0 : job - 3;
    const int N = layer_n(layer);  // 48 or 64
    const __nv_bfloat16* H = layer == 0 ? nullptr : act + (size_t)(layer - 1) * n_max * kWidth;
    const __nv_bfloat16* D = layer == 5 ? gout : delta + (size_t)layer * n_max * kWidth;  // delta_{l+1} at index l
    const int ldD = layer == 5 ? kOut : kWidth;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    float acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[nt][r] = 0.0f;
    for (size_t s0 = c0; s0 < c1; s0 += kDwStage) {
        __syncthreads();
        // stage H (64 records x 64 features; for W0 the job's 64 columns of the encodings) and D
        const __nv_bfloat16* Hs_src = layer == 0 ? enc + 64 * job : H;
        const int ldH = layer == 0 ? kEnc : kWidth;
        for (int i = threadIdx.x; i < kDwStage * 8; i += kThreads) {
            const int r = i >> 3, ch = i & 7;
            const size_t row = s0 + r;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (row < c1) v = *reinterpret_cast<const uint4*>(Hs_src + row * ldH + ch * 8);
            *reinterpret_cast<uint4*>(&Hs[r * kDwLd + ch * 8]) = v;
        }
        const int chunks = ldD / 8;
        for (int i = threadIdx.x; i < kDwStage * chunks; i += kThreads) {
            const int r = i / chunks, ch = i % chunks;
            const size_t row = s0 + r;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (row < c1) v = *reinterpret_cast<const uint4*>(D + row * ldD + ch * 8);
            *reinterpret_cast<uint4*>(&Ds[r * kDwLd + ch * 8]) = v;
        }
        __syncthreads();
        const int m = 16 * warp + g;
#pragma unroll
        for (int k0 = 0; k0 < kDwStage; k0 += 16) {
            auto hp = [&](int k, int mm) { return (uint32_t)Hs[k * kDwLd + mm]; };
            uint32_t a[4];
            a[0] = hp(k0 + 2 * t, m) | (hp(k0 + 2 * t + 1, m) << 16);
            a[1] = hp(k0 + 2 * t, m + 8) | (hp(k0 + 2 * t + 1, m + 8) << 16);
            a[2] = hp(k0 + 2 * t + 8, m) | (hp(k0 + 2 * t + 9, m) << 16);
            a[3] = hp(k0 + 2 * t + 8, m + 8) | (hp(k0 + 2 * t + 9, m + 8) << 16);
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                if (nt < N / 8) {
                    const int nn = 8 * nt + g;
                    uint2 b;
                    b.x = (uint32_t)Ds[(k0 + 2 * t) * kDwLd + nn] | ((uint32_t)Ds[(k0 + 2 * t + 1) * kDwLd + nn] << 16);
                    b.y = (uint32_t)Ds[(k0 + 2 * t + 8) * kDwLd + nn] | ((uint32_t)Ds[(k0 + 2 * t + 9) * kDwLd + nn] << 16);
                    mma_bf16(acc[nt], a, b);
                }
            }
        }
    }
    float* G = grads + param_offset(layer);
    const int mrow = (layer == 0 ? 64 * job : 0) + 16 * warp + g;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        if (nt < N / 8) {
            const int c = 8 * nt + 2 * t;
            atomicAdd(G + (size_t)mrow * N + c, acc[nt][0]);
            atomicAdd(G + (size_t)mrow * N + c + 1, acc[nt][1]);
            atomicAdd(G + (size_t)(mrow + 8) * N + c, acc[nt][2]);
            atomicAdd(G + (size_t)(mrow + 8) * N + c + 1, acc[nt][3]);
        }
    }
}

__global__ void k_adam(float* __restrict__ P, float* __restrict__ Gr, float* __restrict__ M, float* __restrict__ V,
                       const uint32_t* __restrict__ step, float lr, float b1, float b2, float eps, float* grad_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    const float g = Gr[i];
    if (grad_out) grad_out[i] = g;
    Gr[i] = 0.0f;
    if (lr <= 0.0f) return;  // gradients only
    const float t = (float)(*step + 1);
    const float m = b1 * M[i] + (1.0f - b1) * g;
    const float v = b2 * V[i] + (1.0f - b2) * g * g;
    M[i] = m;
    V[i] = v;
    const float mh = m / (1.0f - powf(b1, t)), vh = v / (1.0f - powf(b2, t));
    P[i] -= lr * mh / (sqrtf(vh) + eps);
}

int g_alloc(liar_gpu_ctx* ctx, liar_gpu_guide* G, size_t bytes, void** p, const char* what) {
    cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return ctx_cuda(ctx, e, what);
    }
    G->buffers.push_back(*p);
    return LIAR_OK;
}

int ensure_train_buffers(liar_gpu_ctx* ctx, liar_gpu_guide* G, size_t n) {
    if (G->cap >= n) return LIAR_OK;
    for (void* p : {(void*)G->enc, (void*)G->act, (void*)G->delta, (void*)G->gout}) {
        if (!p) continue;
        cudaFree(p);
        G->buffers.erase(std::remove(G->buffers.begin(), G->buffers.end(), p), G->buffers.end());
    }
    G->enc = G->act = G->delta = G->gout = nullptr;
    G->cap = 0;
    void* p = nullptr;
    int rc = g_alloc(ctx, G, n * kEnc * 2, &p, "guide encodings");
    if (rc) return rc;
    G->enc = static_cast<__nv_bfloat16*>(p);
    rc = g_alloc(ctx, G, n * 5 * kWidth * 2, &p, "guide activations");
    if (rc) return rc;
    G->act = static_cast<__nv_bfloat16*>(p);
    rc = g_alloc(ctx, G, n * 5 * kWidth * 2, &p, "guide deltas");
    if (rc) return rc;
    G->delta = static_cast<__nv_bfloat16*>(p);
    rc = g_alloc(ctx, G, n * kOut * 2, &p, "guide output gradients");
    if (rc) return rc;
    G->gout = static_cast<__nv_bfloat16*>(p);
    G->cap = n;
    return LIAR_OK;
}

int smem_attrs(liar_gpu_ctx* ctx) {
    static int done_device = -1;
    if (done_device == ctx->device) return LIAR_OK;
    cudaError_t e = cudaFuncSetAttribute(k_train_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEvalSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_train_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBwdBytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_eval_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kUmmaSmem);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "guide kernel attributes");
    done_device = ctx->device;
    return LIAR_OK;
}

// host-side initialisation: uniform(-s, s), s = sqrt(6 / fan_in) (He), the output layer x 0.1
void init_params(std::vector<float>& P, uint64_t seed) {
    P.assign(kParams, 0.0f);
    uint64_t state = mix64(seed ^ 0x6a09e667f3bcc909ull);
    auto uni = [&]() {
        state = mix64(state);
        return (float)((state >> 40) * (1.0 / 16777216.0)) * 2.0f - 1.0f;
    };
    for (int l = 0; l < kLayers; ++l) {
        const int K = layer_k(l), N = layer_n(l);
        const int fan_in = l == 0 ? kEncUsed : kWidth;
        const float s = std::sqrt(6.0f / fan_in) * (l == 5 ? 0.1f : 1.0f);
        float* W = P.data() + param_offset(l);
        for (int k = 0; k < K; ++k)
            for (int nn = 0; nn < N; ++nn) {
                const float u = uni();
                const bool pad = (l == 0 && k >= kEncUsed) || (l == 5 && nn >= kOutUsed);
                W[k * N + nn] = pad ? 0.0f : s * u;
            }
    }
}

}  // namespace

namespace liar_gpu {
namespace guide {

int guide_train(liar_gpu_ctx* ctx, liar_gpu_guide* G, const float* d_records, const uint32_t* d_count, size_t n_max,
                int apply, float* d_grad_out, float* d_loss_out, cudaStream_t st) {
    int rc = ensure_train_buffers(ctx, G, n_max);
    if (rc) return rc;
    rc = smem_attrs(ctx);
    if (rc) return rc;
    const Box box = make_box(G->cfg);
    cudaError_t e = cudaMemsetAsync(G->scalars, 0, 2 * sizeof(float), st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "guide scalars");
    const int sms = ctx->num_sms;
    k_weight_sum<<<sms * 4, 256, 0, st>>>(d_records, d_count, n_max, G->scalars);
    const unsigned tiles = (unsigned)((n_max + 31) / 32);
    const unsigned fgrid = std::max(1u, std::min<unsigned>((tiles + kFwdWarps - 1) / kFwdWarps, (unsigned)sms));
    const unsigned grid = std::max(1u, std::min<unsigned>((tiles + 3) / 4, (unsigned)sms * 2));
    k_train_forward<<<fgrid, kFwdThreads, kEvalSmem, st>>>(G->frag_fwd, d_records, d_count, n_max, box, G->scalars, G->enc,
                                                           G->act,
                                                        G->gout, G->scalars + 1);
    k_train_backward<<<grid, kThreads, kBwdBytes, st>>>(G->frag_bwd, d_count, n_max, G->act, G->gout, G->delta);
    const dim3 dwg((unsigned)((n_max + kDwChunk - 1) / kDwChunk), 9);
    k_train_dw<<<dwg, kThreads, 0, st>>>(d_count, n_max, G->enc, G->act, G->delta, G->gout, G->grads);
    const float lr = apply ? (G->cfg.learning_rate > 0 ? G->cfg.learning_rate : 5e-3f) : 0.0f;
    k_adam<<<(kParams + 255) / 256, 256, 0, st>>>(G->params, G->grads, G->adam_m, G->adam_v, G->step, lr, 0.9f, 0.99f,
                                                  1e-8f, d_grad_out);
    if (apply) {
        rc = launch_pack(G, st, 1);
        if (rc) return ctx_cuda(ctx, cudaGetLastError(), "guide pack");
        G->steps_done += 1;
    }
    if (d_loss_out) {
        e = cudaMemcpyAsync(d_loss_out, G->scalars + 1, sizeof(float), cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "guide loss");
    }
    return ctx_cuda(ctx, cudaGetLastError(), "guide training launch");
}

}  // namespace guide
}  // namespace liar_gpu

// ---- C ABI

extern "C" size_t liar_gpu_guide_param_count(void) { return (size_t)kParams; }

extern "C" int liar_gpu_guide_create(liar_gpu_ctx* ctx, const liar_guide_config* cfg, liar_gpu_guide** out) {
    if (!ctx || !cfg || !out) return LIAR_ERR_INVALID;
    *out = nullptr;
    for (int k = 0; k < 3; ++k)
        if (!(cfg->bounds_hi[k] > cfg->bounds_lo[k]) || !std::isfinite(cfg->bounds_lo[k]) || !std::isfinite(cfg->bounds_hi[k]))
            return ctx_fail(ctx, LIAR_ERR_INVALID, "guide bounds must be finite with hi > lo");
    if (cfg->guide_probability < 0.0f || cfg->guide_probability >= 1.0f)
        return ctx_fail(ctx, LIAR_ERR_INVALID, "guide_probability must lie in [0, 1)");
    if (cfg->light_probability < 0.0f || cfg->light_probability >= 1.0f)
        return ctx_fail(ctx, LIAR_ERR_INVALID, "light_probability must lie in [0, 1)");
    if (cfg->learning_rate < 0.0f || cfg->batch_records < 0 || cfg->steps_per_pass < 0)
        return ctx_fail(ctx, LIAR_ERR_INVALID, "negative learning rate, batch or step count");
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    liar_gpu_guide* G = new (std::nothrow) liar_gpu_guide();
    if (!G) return ctx_fail(ctx, LIAR_ERR_OOM, "host allocation");
    G->device = ctx->device;
    G->cfg = *cfg;
    void* p = nullptr;
    rc = g_alloc(ctx, G, 4 * (size_t)kParams * sizeof(float) + 256, &p, "guide parameters");
    if (!rc) {
        float* f = static_cast<float*>(p);
        G->params = f;
        G->grads = f + kParams;
        G->adam_m = f + 2 * kParams;
        G->adam_v = f + 3 * kParams;
        G->step = reinterpret_cast<uint32_t*>(f + 4 * kParams);
        G->scalars = f + 4 * kParams + 4;
    }
    if (!rc) rc = g_alloc(ctx, G, kFwdBytes, &p, "guide fragments");
    if (!rc) G->frag_fwd = static_cast<uint2*>(p);
    if (!rc) rc = g_alloc(ctx, G, kBwdBytes, &p, "guide fragments");
    if (!rc) G->frag_bwd = static_cast<uint2*>(p);
    if (!rc) rc = g_alloc(ctx, G, kUmmaWBytes, &p, "guide operand images");
    if (!rc) G->umma_w = static_cast<unsigned char*>(p);
    if (!rc) {
        std::vector<float> P;
        init_params(P, cfg->seed);
        cudaError_t e = cudaMemcpy(G->params, P.data(), kParams * sizeof(float), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemset(G->grads, 0, 3 * (size_t)kParams * sizeof(float) + 256);
        if (e != cudaSuccess) rc = ctx_cuda(ctx, e, "guide initialisation");
    }
    if (!rc && launch_pack(G, ctx->stream, 0)) rc = ctx_cuda(ctx, cudaGetLastError(), "guide pack");
    if (!rc) rc = ctx_cuda(ctx, cudaStreamSynchronize(ctx->stream), "guide initialisation");
    if (rc) {
        liar_gpu_guide_destroy(G);
        return rc;
    }
    *out = G;
    return LIAR_OK;
}

extern "C" void liar_gpu_guide_destroy(liar_gpu_guide* G) {
    if (!G) return;
    int cur = -1;
    cudaGetDevice(&cur);
    if (G->device >= 0) cudaSetDevice(G->device);
    for (void* p : G->buffers) cudaFree(p);
    if (cur >= 0) cudaSetDevice(cur);
    delete G;
}

extern "C" int liar_gpu_guide_get_params(liar_gpu_ctx* ctx, const liar_gpu_guide* G, float* host, size_t n) {
    if (!ctx || !G || !host) return LIAR_ERR_INVALID;
    if (n != (size_t)kParams) return ctx_fail(ctx, LIAR_ERR_INVALID, "expected %d parameters", kParams);
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpy(host, G->params, n * sizeof(float), cudaMemcpyDeviceToHost);
    return ctx_cuda(ctx, e, "guide parameters");
}

extern "C" int liar_gpu_guide_set_params(liar_gpu_ctx* ctx, liar_gpu_guide* G, const float* host, size_t n) {
    if (!ctx || !G || !host) return LIAR_ERR_INVALID;
    if (n != (size_t)kParams) return ctx_fail(ctx, LIAR_ERR_INVALID, "expected %d parameters", kParams);
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(host[i])) return ctx_fail(ctx, LIAR_ERR_INVALID, "parameter %zu is not finite", i);
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpy(G->params, host, n * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(G->grads, 0, 3 * (size_t)kParams * sizeof(float) + 256);  // grads, Adam, step
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "guide parameters");
    if (launch_pack(G, ctx->stream, 0)) return ctx_cuda(ctx, cudaGetLastError(), "guide pack");
    G->steps_done = 0;
    G->records = G->guided = G->passes = 0;
    return ctx_cuda(ctx, cudaStreamSynchronize(ctx->stream), "guide parameters");
}

namespace liar_gpu {
namespace guide {
int guide_eval(liar_gpu_ctx* ctx, const liar_gpu_guide* G, const float* d_inputs, size_t n, float* d_mixture,
               int stride, cudaStream_t st);
}  // namespace guide
}  // namespace liar_gpu

extern "C" int liar_gpu_guide_eval_device(liar_gpu_ctx* ctx, const liar_gpu_guide* G, const float* d_inputs, size_t n,
                                          float* d_mixture, void* stream) {
    if (!ctx) return LIAR_ERR_INVALID;
    return guide_eval(ctx, G, d_inputs, n, d_mixture, kOutUsed, stream ? (cudaStream_t)stream : ctx->stream);
}

// inference: raw inputs [n][9] -> mixtures [n][stride] = 8 x (mu xyz, kappa), the 8 weights and,
// with stride kMixRender, the 8 weights times their lobe's normalisation
int liar_gpu::guide::guide_eval(liar_gpu_ctx* ctx, const liar_gpu_guide* G, const float* d_inputs, size_t n,
                                float* d_mixture, int stride, cudaStream_t st) {
    if (!ctx || !G) return LIAR_ERR_INVALID;
    if (n == 0) return LIAR_OK;
    if (!d_inputs || !d_mixture) return ctx_fail(ctx, LIAR_ERR_INVALID, "null inputs or outputs");
    if (G->device != ctx->device) return ctx_fail(ctx, LIAR_ERR_INVALID, "guide lives on another device");
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    rc = smem_attrs(ctx);
    if (rc) return rc;
    if (stride != kOutUsed && stride != kMixRender) return ctx_fail(ctx, LIAR_ERR_INVALID, "mixture stride %d", stride);
    const size_t tiles = (n + kTcRows - 1) / kTcRows;
    const unsigned grid = (unsigned)std::max<size_t>(1, std::min<size_t>((tiles + kTcSlots - 1) / kTcSlots, (size_t)ctx->num_sms));
    // the bounded waits' limit: 2^24 polls, far beyond a layer's MMAs; the timeout test
    // (liar_gpu_set_fault_test) issues no MMA and gives up after 2^16 polls
    const bool wait_test = ctx->fault_test == LIAR_FAULT_TEST_GUIDE_WAIT;
    k_eval_tc<<<grid, kTcThreads, kUmmaSmem, st>>>(G->umma_w, d_inputs, n, make_box(G->cfg), d_mixture, stride,
                                                   ctx->d_scratch + kStatusWord, wait_test ? 1u << 16 : 1u << 24,
                                                   wait_test ? 0 : 1);
    return ctx_cuda(ctx, cudaGetLastError(), "guide evaluation");
}

extern "C" int liar_gpu_guide_train_device(liar_gpu_ctx* ctx, liar_gpu_guide* G, const float* d_records, size_t n,
                                           int apply, float* d_grad, float* d_loss, void* stream) {
    if (!ctx || !G) return LIAR_ERR_INVALID;
    if (n == 0) return LIAR_OK;
    if (!d_records) return ctx_fail(ctx, LIAR_ERR_INVALID, "null records");
    if (n > (1u << 24)) return ctx_fail(ctx, LIAR_ERR_INVALID, "at most 2^24 records per step");
    if (G->device != ctx->device) return ctx_fail(ctx, LIAR_ERR_INVALID, "guide lives on another device");
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    return guide_train(ctx, G, d_records, nullptr, n, apply, d_grad, d_loss, stream ? (cudaStream_t)stream : ctx->stream);
}

namespace {
__global__ void k_sample(const float* __restrict__ mix, const float* __restrict__ u, size_t n, float* __restrict__ dirs,
                         float* __restrict__ pdf) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float m[kOutUsed];
    for (int c = 0; c < kOutUsed; ++c) m[c] = mix[i * kOutUsed + c];
    float dx, dy, dz;
    mixture_sample(m, u[3 * i], u[3 * i + 1], u[3 * i + 2], dx, dy, dz);
    dirs[3 * i] = dx;
    dirs[3 * i + 1] = dy;
    dirs[3 * i + 2] = dz;
    pdf[i] = mixture_pdf(m, dx, dy, dz);
}
}  // namespace

extern "C" int liar_gpu_guide_sample_device(liar_gpu_ctx* ctx, const float* d_mixture, const float* d_u, size_t n,
                                            float* d_dirs, float* d_pdf, void* stream) {
    if (!ctx) return LIAR_ERR_INVALID;
    if (n == 0) return LIAR_OK;
    if (!d_mixture || !d_u || !d_dirs || !d_pdf) return ctx_fail(ctx, LIAR_ERR_INVALID, "null buffer");
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    k_sample<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_mixture, d_u, n, d_dirs, d_pdf);
    return ctx_cuda(ctx, cudaGetLastError(), "mixture sampling");
}

extern "C" int liar_gpu_guide_stats(const liar_gpu_guide* G, unsigned long long* out4) {
    if (!G || !out4) return LIAR_ERR_INVALID;
    out4[0] = G->steps_done;
    out4[1] = G->records;
    out4[2] = G->guided;
    out4[3] = G->passes;
    return LIAR_OK;
}
