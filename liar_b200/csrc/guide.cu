// guide.cu -- the path-guiding network: inference, online training (Adam), and its C ABI
// (no reference counterpart; the reference's AdjointPhotonTracer samples BSDF and lights only,
// src/liar/tracers/adjoint_photon_tracer.cpp:212-292).
//
// Training minimises the KL divergence from the normalised integrand to the guide
// (neural importance sampling, Mueller et al. 2019): for records (x, w, F/p) the loss is
//   L = -(1/B) sum_i min((F_i/p_i) / mean(F/p), 20) * log q(w_i | x_i),
// q = sum_l pi_l vMF(w; mu_l, kappa_l), pi = softmax(logits), mu = m / |m|, kappa = e^{clamp(s)}.
// One step, every GEMM on the 5th-generation tensor cores (tcgen05): forward (stores the bf16
// activations and the output gradient, fused) -> backward (stores the bf16 layer deltas) -> weight
// gradients over the records (TMA-fed), accumulated in tensor memory as per-CTA partial sums ->
// their sum, Adam on the f32 master weights and the repacked bf16 operand images, one kernel.
#include <cuda.h>
#include <cudaTypedefs.h>
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
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    unsigned char* umma_w = nullptr;   // forward B-operand images of the six layers (inference, training)
    unsigned char* umma_wb = nullptr;  // backward B-operand images of W1..W5 (training)
    // training scratch, sized for cap records
    size_t cap = 0;
    __nv_bfloat16* act = nullptr;    // h_1..h_5: [5][cap][64]
    __nv_bfloat16* delta = nullptr;  // delta_1..delta_5: [5][cap][64]
    __nv_bfloat16* gout = nullptr;   // [cap][48]
    float* grad_part = nullptr;      // [part_cap][kParams]: the weight-gradient CTAs' partial sums
    float* wpart = nullptr;          // [kWeightParts]: k_weight_sum's block sums
    int part_cap = 0;
    float* scalars = nullptr;        // [1] the step's loss sum ([0] unused)
    // TMA descriptors of act, delta and gout for the weight-gradient kernel, for tm_rows records
    CUtensorMap tm_act{}, tm_delta{}, tm_gout{};
    // TMA descriptors through which the forward and backward store their activation / delta tiles
    CUtensorMap tm_act_st{}, tm_delta_st{};
    const void* tm_base = nullptr;
    size_t tm_rows = 0;
    std::vector<void*> buffers;
    unsigned long long steps_done = 0;
    unsigned long long records = 0, guided = 0, passes = 0;
};

namespace liar_gpu {
namespace guide {
// used by the guided renderer (guided.cu)
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

constexpr int kRecordFloats = 13;
// normalised record weights are clipped here: radiance estimates are heavy-tailed and a handful of
// records would otherwise set the whole gradient (the renderer stays unbiased whatever the guide)
constexpr float kWeightClip = 20.0f;
constexpr int kWeightParts = 1024;  // most blocks of k_weight_sum (one sum each)
// rows per layer of the training activations and deltas ([5][act_rows(n)][64] bf16): n rounded up
// to whole 8-row groups, the unit the tile stores write
__host__ __device__ __forceinline__ size_t act_rows(size_t n) { return (n + 7) & ~(size_t)7; }

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

// ---- operand images

// backward B images: layer l (1..5) element (n, k) = W_l[n][k] at umma_offset(n, k, N_l)
__host__ __device__ constexpr uint32_t umma_wb_offset(int l) { return 8192u * (uint32_t)(l - 1); }
constexpr uint32_t kUmmaWbBytes = 4u * 8192u + 6144u;  // W1..W4 64 x 64, W5 64 x 48


// the tcgen05 B operands: layer l's element (n, k) = W_l[k][n] at umma_offset(n, k, K_l) in img
// (the forward), and for l >= 1 element (k, n) at umma_offset(k, n, N_l) in img_b (the backward,
// W_l transposed): parameter i (row-major [in][out] within its layer) as bf16 into both
__device__ __forceinline__ void pack_param(int i, float value, unsigned char* __restrict__ img,
                                           unsigned char* __restrict__ img_b) {
    int l = 0;
    while (l < 5 && i >= param_offset(l + 1)) ++l;
    const int loc = i - param_offset(l), N = layer_n(l), K = layer_k(l);
    const int k = loc / N, n = loc % N;
    const __nv_bfloat16 w = __float2bfloat16_rn(value);
    *reinterpret_cast<__nv_bfloat16*>(img + umma_w_offset(l) + umma_offset((uint32_t)n, (uint32_t)k, (uint32_t)K)) = w;
    if (l >= 1)
        *reinterpret_cast<__nv_bfloat16*>(img_b + umma_wb_offset(l) + umma_offset((uint32_t)k, (uint32_t)n, (uint32_t)N)) = w;
}
__global__ void k_pack_umma(const float* __restrict__ P, unsigned char* __restrict__ img, unsigned char* __restrict__ img_b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;  // one parameter (k, n) per thread
    if (i < kParams) pack_param(i, P[i], img, img_b);
}

// the loss gradient of one record with respect to the 40 raw outputs (scaled by `scale`); the
// mixture from mixture_head_fast, the hardware's approximate exponential, logarithm and division
// (relative errors of a few 1e-7, far below the bf16 rounding of the gradient), expm1f where
// 1 - e^{-2 kappa} cancels
__device__ float record_gradient(const float* o, float wx, float wy, float wz, float weight, float scale, float* d);


// The inference head: mixture_from_raw with the hardware's approximate reciprocal square root,
// exponential and division (relative errors of a few 1e-7, far below the bf16 rounding of the
// network), and each lobe's weight times its vMF normalisation for the renderer's copy.
__device__ __forceinline__ void mixture_head_fast(const float* o, Lobe* lobes, float* w) {
    float mx = -3.0e38f;
#pragma unroll
    for (int l = 0; l < kLobes; ++l) mx = fmaxf(mx, o[5 * l + 4]);
    float sum = 0.0f;
#pragma unroll
    for (int l = 0; l < kLobes; ++l) {
        const float x = o[5 * l], y = o[5 * l + 1], z = o[5 * l + 2];
        const float n2 = x * x + y * y + z * z;
        if (n2 > 0.0f) {
            const float inv = rsqrtf(n2);
            lobes[l].mx = x * inv;
            lobes[l].my = y * inv;
            lobes[l].mz = z * inv;
        } else {
            lobes[l].mx = lobes[l].my = 0.0f;
            lobes[l].mz = 1.0f;
        }
        lobes[l].kappa = __expf(fminf(fmaxf(o[5 * l + 3], kLogKappaMin), kLogKappaMax));
        w[l] = __expf(o[5 * l + 4] - mx);
        sum += w[l];
    }
    const float inv_sum = __fdividef(1.0f, sum);
#pragma unroll
    for (int l = 0; l < kLobes; ++l) w[l] *= inv_sum;
}
__device__ __forceinline__ float vmf_norm_fast(float kappa) {
    return __fdividef(kappa, 6.283185307179586f * -expm1f(-2.0f * kappa));
}

__device__ float record_gradient(const float* o, float wx, float wy, float wz, float weight, float scale, float* d) {
    Lobe L[kLobes];
    float pi[kLobes], la[kLobes], cs[kLobes];
    mixture_head_fast(o, L, pi);
    float mx = -3.0e38f;
    for (int l = 0; l < kLobes; ++l) {
        cs[l] = L[l].mx * wx + L[l].my * wy + L[l].mz * wz;
        la[l] = __logf(pi[l]) + __logf(__fdividef(L[l].kappa, -expm1f(-2.0f * L[l].kappa))) -
                1.8378770664093453f /* log 2 pi */ + L[l].kappa * (cs[l] - 1.0f);
        mx = fmaxf(mx, la[l]);
    }
    float s = 0.0f;
    for (int l = 0; l < kLobes; ++l) s += __expf(la[l] - mx);
    const float lq = mx + __logf(s);
    const float ws = weight * scale;
    for (int l = 0; l < kLobes; ++l) {
        const float r = __expf(la[l] - lq);
        const float k = L[l].kappa;
        const float c = -ws * r;
        d[5 * l + 4] = -ws * (r - pi[l]);
        const float sk = o[5 * l + 3];
        d[5 * l + 3] = (sk > kLogKappaMin && sk < kLogKappaMax) ? c * k * (__fdividef(1.0f, k) - __fdividef(2.0f, expm1f(2.0f * k)) + cs[l] - 1.0f)
                                                                 : 0.0f;
        // d mu / d m = (I - mu mu^T) / |m|
        const float nm = sqrtf(o[5 * l] * o[5 * l] + o[5 * l + 1] * o[5 * l + 1] + o[5 * l + 2] * o[5 * l + 2]);
        const float f = __fdividef(c * k, fmaxf(nm, kMeanNormMin));
        d[5 * l + 0] = f * (wx - cs[l] * L[l].mx);
        d[5 * l + 1] = f * (wy - cs[l] * L[l].my);
        d[5 * l + 2] = f * (wz - cs[l] * L[l].mz);
    }
    return -weight * lq;
}

// ---- inference on tcgen05: four slots of 128 rows per CTA (guide_umma.cuh)
// Layer 0 runs as four K-chunks over the two halves of the slot's buffer, each chunk committed to
// the half's own mbarrier; a half is rewritten only after the commit of the chunk that read it.
// Every mbarrier wait is bounded by max_tries polls. A wait that runs out records the timeout,
// waits once more (bounded again) for every commit still outstanding, so that no MMA still writes
// the accumulator, and the CTA frees its TMEM and leaves. issue_mma = 0 is the timeout test: no
// MMA and no commit are issued, so the first wait runs out with nothing in flight.
// Inference writes each row's mixture (stride floats) through tm_store, a 2D map over the
// [n][stride] output. TRAIN (the training forward): the inputs are training records (13 floats, the
// first 9 the network's inputs), the row count may come from device memory (n_dev, at most n),
// every hidden layer's bf16 activations h_1..h_5 also go to the activation buffer
// ([5][act_rows(n_max)][64]) through tm_store (then a 5D map of the tile stores), and the output layer ends in the loss head instead
// of the mixture: each row's loss gradient with respect to its 40 raw outputs (record_gradient,
// weights normalised by the batch mean from k_weight_sum's block sums, clipped) goes to gout as
// 48 bf16 (the last 8 zero), the batch loss is added to train[1].
template <bool TRAIN>
__global__ void __launch_bounds__(kEvThreads, 1) k_eval_tc(const unsigned char* __restrict__ w_img,
                                                           const float* __restrict__ in, size_t n, Box box,
                                                           int stride,
                                                           uint32_t* __restrict__ status, uint32_t max_tries,
                                                           int issue_mma, const uint32_t* __restrict__ n_dev,
                                                           size_t n_max, float* __restrict__ train,
                                                           __nv_bfloat16* __restrict__ gout,
                                                           const float* __restrict__ wpart, int n_wpart,
                                                           const __grid_constant__ CUtensorMap tm_store) {
    constexpr int IN = TRAIN ? kRecordFloats : kIn;
    if (TRAIN && n_dev) n = min((size_t)*n_dev, n);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char* sw = smem;
    uint64_t* mbar_all = reinterpret_cast<uint64_t*>(sw + kUmmaWBytes + (size_t)kEvSlots * (kEvBuf + kEvIn));
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar_all + 2 * kEvSlots);
    volatile uint32_t* failed = tmem_slot + 1;  // one flag per slot
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    const uint32_t slot = tid >> 7, r = tid & 127u;  // this thread's slot and row within the slot's tile
    unsigned char* buf = sw + kUmmaWBytes + slot * kEvBuf;
    float* stage_in = reinterpret_cast<float*>(sw + kUmmaWBytes + (size_t)kEvSlots * kEvBuf + slot * kEvIn);
    {
        const uint4* s = reinterpret_cast<const uint4*>(w_img);
        uint4* d = reinterpret_cast<uint4*>(sw);
        for (uint32_t i = tid; i < kUmmaWBytes / 16; i += kEvThreads) d[i] = s[i];
    }
    if (tid == 0) {
        for (int k = 0; k < 2 * kEvSlots; ++k)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((uint32_t)__cvta_generic_to_shared(mbar_all + k)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        for (int k = 0; k < kEvSlots; ++k) failed[k] = 0u;
    }
    if (warp == 0) {
        const uint32_t sa = (uint32_t)__cvta_generic_to_shared(tmem_slot);
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sa), "r"(kEvTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // the training forward follows k_weight_sum (programmatic launch): the prologue above ran
    // beside it, its weight sum is read after the wait
    grid_dependency_wait();
    launch_dependents();
    float inv_mean = 0.0f, inv_b = 0.0f;  // TRAIN: 1 / mean record weight, 1 / batch size
    if (TRAIN) {
        // the weight sum: k_weight_sum's block sums added in one fixed order (lane j takes every
        // 32nd, then a shuffle tree), lane 0's result broadcast, so every thread of every CTA has
        // the same bits
        float wsum = 0.0f;
        for (int j = (int)(tid & 31u); j < n_wpart; j += 32) wsum += wpart[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) wsum += __shfl_down_sync(0xffffffffu, wsum, o);
        wsum = __shfl_sync(0xffffffffu, wsum, 0);
        inv_mean = (wsum > 0.0f && n > 0) ? (float)n / wsum : 0.0f;
        inv_b = n > 0 ? 1.0f / (float)n : 0.0f;
    }
    const uint32_t tmem = *tmem_slot + 64u * slot;              // the slot's accumulator columns
    const uint32_t taddr = tmem + ((32u * (warp & 3u)) << 16);  // the warp's lane quarter
    const uint32_t mb[2] = {(uint32_t)__cvta_generic_to_shared(mbar_all + 2 * slot),
                            (uint32_t)__cvta_generic_to_shared(mbar_all + 2 * slot + 1)};
    const uint32_t sw_addr = (uint32_t)__cvta_generic_to_shared(sw);
    const uint32_t buf_addr = (uint32_t)__cvta_generic_to_shared(buf);
    auto slot_sync = [&]() { asm volatile("bar.sync %0, 128;" ::"r"(1u + slot) : "memory"); };
    uint32_t phase[2] = {0u, 0u};
    bool pending[2] = {false, false};  // a commit to the half's mbarrier not yet waited for
    // wait for half h's outstanding commit. Every thread polls the mbarrier itself, so no barrier
    // follows: a thread that gives up marks the slot failed and keeps the commit pending (the drain
    // waits for it again), and the whole slot sees the mark at the barrier of its next issue
    auto wait_half = [&](int h) {
        if (mbar_wait(mb[h], phase[h], max_tries)) {
            phase[h] ^= 1u;
            pending[h] = false;
        } else {
            failed[slot] = 1u;
        }
    };
    // hand the slot's operand to the tensor core (the writes of every thread are visible to the
    // async proxy and the accumulator reads are done) and, from thread 0, issue K / 16 MMAs; false
    // (for the whole slot, nothing issued) once a wait of the slot has given up
    auto issue = [&](uint32_t a_addr, uint32_t a_sbo, uint32_t b_addr, uint32_t b_sbo, uint32_t ksteps, uint32_t N,
                     bool acc0, int h) -> bool {
        fence_async_smem();
        tc_fence_before();
        slot_sync();
        tc_fence_after();
        if (failed[slot]) return false;
        if (r == 0 && issue_mma) {
            const uint32_t idesc = umma_idesc(N);
            for (uint32_t j = 0; j < ksteps; ++j)
                umma_bf16(tmem, umma_smem_desc(a_addr + 256u * j, a_sbo), umma_smem_desc(b_addr + 256u * j, b_sbo), idesc,
                          (acc0 || j > 0) ? 1u : 0u);
            umma_commit(mb[h]);
        }
        pending[h] = true;
        return true;
    };
    const size_t n_tiles = (n + kTcRows - 1) / kTcRows;
    const size_t tile_step = (size_t)gridDim.x * kEvSlots;
    bool ok = true;
    // the inputs of a tile, coalesced: thread r holds elements r + 128 j (j < IN) of the tile's
    // rows * IN floats; the next tile's are loaded while the current one runs
    float pre[IN];
    auto prefetch = [&](size_t t) {
        const size_t base = t * kTcRows * (size_t)IN, end = min(n * (size_t)IN, base + (size_t)kTcRows * IN);
#pragma unroll
        for (int j = 0; j < IN; ++j) {
            const size_t i = base + r + 128u * (uint32_t)j;
            pre[j] = (t < n_tiles && i < end) ? __ldg(in + i) : 0.0f;
        }
    };
    prefetch((size_t)blockIdx.x * kEvSlots + slot);
    for (size_t tile = (size_t)blockIdx.x * kEvSlots + slot; ok && tile < n_tiles; tile += tile_step) {
        const size_t row0 = tile * kTcRows;
        const uint32_t rows = n - row0 < (size_t)kTcRows ? (uint32_t)(n - row0) : (uint32_t)kTcRows;
        // the tile's inputs through shared memory (the previous tile's readers have passed the slot
        // barriers since), then the next tile's loads go out
#pragma unroll
        for (int j = 0; j < IN; ++j) stage_in[r + 128u * (uint32_t)j] = pre[j];
        prefetch(tile + tile_step);
        if (r == 0) bulk_wait_read();  // the previous tile's last store has read its buffer
        slot_sync();
        float x[kIn];
        if (r < rows) normalise_input(stage_in + r * IN, box.lo, box.inv_ext, x);
        else
            for (int c = 0; c < kIn; ++c) x[c] = 0.0f;
        // layer 0: chunk c's encodings into half c % 2 once the chunk before last has been consumed
        uint32_t carry[8];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int h = c & 1;
            if (c >= 2) wait_half(h);
            encode_chunk_carry(x, buf + h * kEvHalf, r, c, carry);
            if (!issue(buf_addr + h * kEvHalf, 1024u, sw_addr + umma_w_offset(0) + 1024u * c, (kEnc / 8) * 128u, 4u,
                       kWidth, c > 0, h)) {
                ok = false;
                break;
            }
        }
        if (ok) {
            wait_half(0);
            wait_half(1);
        }
        // hidden layers and the output layer from half 0
        for (int l = 1; ok && l <= kLayers; ++l) {
            tc_fence_after();
            // training alternates the hidden layers between the halves (h_l in half l % 2), so that
            // the TMA store of one layer's operand runs on while the next layer's is written
            const uint32_t hh = TRAIN ? (uint32_t)(l & 1) * kEvHalf : 0u;
            unsigned char* dst = buf + hh + (r >> 3) * (kWidth / 8) * 128u + (r & 7u) * 16u;
            if (l < kLayers) {
                // ReLU, bf16, the next layer's A operand (row r, 8 chunks of 8 columns)
                {
                    float v[64];
                    tmem_ld_x64(taddr, v);
#pragma unroll
                    for (int c = 0; c < 8; ++c) {
                        const float* q = v + 8 * c;
                        // training: rows past the record count hold zeros (they leave with the tile;
                        // their MMA outputs are never read)
                        const uint4 hq = (!TRAIN || r < rows)
                                             ? make_uint4(pack_bf16_relu(q[0], q[1]), pack_bf16_relu(q[2], q[3]),
                                                          pack_bf16_relu(q[4], q[5]), pack_bf16_relu(q[6], q[7]))
                                             : make_uint4(0u, 0u, 0u, 0u);
                        *reinterpret_cast<uint4*>(dst + c * 128u) = hq;
                    }
                }
                // training: the previous layer's store has read the other half before the barrier,
                // after which that half may be rewritten (by layer l + 1, or by the loss head's rows)
                if (TRAIN && r == 0) bulk_wait_read();
                if (!issue(buf_addr + hh, (kWidth / 8) * 128u, sw_addr + umma_w_offset(l), (kWidth / 8) * 128u, kWidth / 16,
                           (uint32_t)layer_n(l), false, 0)) {
                    ok = false;
                    break;
                }
                // training: h_l leaves the operand by one TMA store while the layer's MMAs read it (the
                // tile's 16 8-row groups, rows past the record count as zeros: the weight-gradient
                // kernel reads whole 32-record stages)
                if (TRAIN && r == 0) tma_store_5d(&tm_store, 0, 0, 0, (int)(row0 >> 3), l - 1, buf_addr + hh);
                wait_half(0);
            } else {
                float o[kOutUsed];
                tmem_ld_32x32b<32>(taddr, o);
                tmem_ld_32x32b<8>(taddr + 32u, o + 32);
                if (TRAIN) {
                    // the loss head: row r's gradient as 48 bf16 (96 B) into the staging rows, the
                    // loss summed per warp, then the slot's gradient rows leave as one coalesced block
                    float lsum = 0.0f;
                    uint4* grow = reinterpret_cast<uint4*>(buf + r * (kOut * 2));
                    if (r >= rows) {  // zero gradient rows to the tile's end (whole weight-gradient stages)
#pragma unroll
                        for (int c = 0; c < kOut / 8; ++c) grow[c] = make_uint4(0u, 0u, 0u, 0u);
                    } else {
                        const float* rr = stage_in + r * IN;
                        float weight = rr[12];
                        if (!(weight > 0.0f) || !isfinite(weight)) weight = 0.0f;
                        float d[kOut];
#pragma unroll
                        for (int c = kOutUsed; c < kOut; ++c) d[c] = 0.0f;
                        lsum = record_gradient(o, rr[9], rr[10], rr[11], fminf(weight * inv_mean, kWeightClip), inv_b, d);
#pragma unroll
                        for (int c = 0; c < kOut / 8; ++c)
                            grow[c] = make_uint4(pack_bf16(d[8 * c], d[8 * c + 1]), pack_bf16(d[8 * c + 2], d[8 * c + 3]),
                                                 pack_bf16(d[8 * c + 4], d[8 * c + 5]), pack_bf16(d[8 * c + 6], d[8 * c + 7]));
                    }
#pragma unroll
                    for (int s = 16; s > 0; s >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, s);
                    if ((tid & 31u) == 0 && lsum != 0.0f) atomicAdd(train + 1, lsum * inv_b);
                    slot_sync();
                    if (failed[slot]) {  // the last layer's wait gave up: nothing leaves
                        ok = false;
                        break;
                    }
                    const uint4* srows = reinterpret_cast<const uint4*>(buf);
                    uint4* gdst = reinterpret_cast<uint4*>(gout + row0 * kOut);
                    const uint32_t rows_out = (uint32_t)min((size_t)kTcRows, n_max - row0);
                    for (uint32_t i = r; i < rows_out * (kOut * 2 / 16); i += 128u) gdst[i] = srows[i];
                } else {
                // the mixture of row r into the staging rows (dense, stride floats per row), then the
                // slot's rows leave by one TMA store of the block (rows past n are not written)
                float* srow = reinterpret_cast<float*>(buf) + r * (uint32_t)stride;
                Lobe lobes[kLobes];
                float w[kLobes];
                mixture_head_fast(o, lobes, w);
#pragma unroll
                for (int k = 0; k < kLobes; ++k)
                    *reinterpret_cast<float4*>(srow + 4 * k) = make_float4(lobes[k].mx, lobes[k].my, lobes[k].mz, lobes[k].kappa);
                *reinterpret_cast<float4*>(srow + 32) = make_float4(w[0], w[1], w[2], w[3]);
                *reinterpret_cast<float4*>(srow + 36) = make_float4(w[4], w[5], w[6], w[7]);
                if (stride == kMixRender) {
                    float a[kLobes];
#pragma unroll
                    for (int k = 0; k < kLobes; ++k) a[k] = w[k] * vmf_norm_fast(lobes[k].kappa);
                    *reinterpret_cast<float4*>(srow + 40) = make_float4(a[0], a[1], a[2], a[3]);
                    *reinterpret_cast<float4*>(srow + 44) = make_float4(a[4], a[5], a[6], a[7]);
                }
                fence_async_smem();
                slot_sync();
                if (failed[slot]) {  // the last layer's wait gave up: nothing leaves
                    ok = false;
                    break;
                }
                if (r == 0) tma_store_2d(&tm_store, 0, (int)row0, buf_addr);
                }
            }
        }
    }
    if (!ok && issue_mma) {
        // drain: the commits this slot gave up on, before the TMEM is freed
        for (int h = 0; h < 2; ++h)
            if (pending[h]) mbar_wait(mb[h], phase[h], max_tries);
    }
    if (r == 0) bulk_wait_all();  // the tile stores are complete before the grid ends
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*tmem_slot), "r"(kEvTmemCols));
    if (tid == 0) {
        uint32_t f = 0;
        for (int k = 0; k < kEvSlots; ++k) f |= failed[k];
        if (f) atomicOr(status, kStatusTimeout);
    }
}

// ---- training

// the batch's record weights (positive and finite ones), one sum per block into wpart; the
// training forward adds the block sums in a fixed order, so that a step is reproducible
__global__ void k_weight_sum(const float* __restrict__ rec, const uint32_t* __restrict__ n_dev, size_t n_max,
                             float* __restrict__ wpart, float* __restrict__ loss) {
    grid_dependency_wait();  // the records and the previous step are complete
    launch_dependents();     // the training forward's prologue reads nothing written here
    if (blockIdx.x == 0 && threadIdx.x == 0) *loss = 0.0f;  // the forward adds the batch's loss after its wait
    const size_t n = n_dev ? min((size_t)*n_dev, n_max) : n_max;
    float s = 0.0f;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float w = rec[i * kRecordFloats + 12];
        if (w > 0.0f && isfinite(w)) s += w;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    __shared__ float warp_sum[32];
    if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float b = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b += warp_sum[w];
        wpart[blockIdx.x] = b;
    }
}


// ---- training on tcgen05 (guide_umma.cuh's operand layouts and instruction forms)
//
// forward  k_eval_tc<true>: the inference kernel's four 4-warp slots of 128 records; after every
//          hidden layer its ReLU'd bf16 activations also go to global memory (h_1..h_5, for the
//          backward masks and the weight gradients); its output layer ends in the loss head (the
//          loss and its gradient per record, record_gradient), stored bf16
// backward k_train_bwd_tc: delta_l = (delta_{l+1} W_l^T) * [h_l > 0] for l = 5..1 (delta_6 =
//          the output gradient), one UMMA chain per 128-record tile with the weights as B
//          operands element (n, k) = W_l[n][k] (n an input, k an output of layer l); each delta
//          is stored bf16 and written back as the next A operand
// weights  k_train_dw_tc: dW_l = H_l^T D_l summed over the records (H_0 the encodings, recomputed;
//          H_l = h_l; D_l = delta_{l+1}, D_5 the output gradient): the records are the K
//          dimension, so each 64-record stage is staged row-major and transposed into K-major
//          operands (A: features x records, B: outputs x records); a CTA accumulates all six
//          weight gradients of its records in tensor memory (448 of 512 columns; the 64-feature
//          layers use the lower half of M = 128, the upper half zero) and adds them to the
//          global gradient once
// Every mbarrier wait is bounded (max_tries polls): a wait that runs out records kStatusTimeout,
// waits once more (bounded) for the commit it gave up on, and the CTA frees its tensor memory.
// issue_mma = 0 (the fault test) issues no MMA or commit, so the first wait runs out.

// the shared prologue of the per-tile kernels (SLOTS 4-warp slots): weights to shared memory,
// mbarriers, TMEM (64 columns per slot)
struct TcTile {
    uint64_t* mbar_all;
    uint32_t* tmem_slot;
    volatile uint32_t* failed;
};
template <int SLOTS>
__device__ __forceinline__ TcTile tc_setup(unsigned char* smem, size_t w_bytes, size_t buf_bytes,
                                           const unsigned char* __restrict__ w_img) {
    TcTile T;
    T.mbar_all = reinterpret_cast<uint64_t*>(smem + w_bytes + (size_t)SLOTS * buf_bytes);
    T.tmem_slot = reinterpret_cast<uint32_t*>(T.mbar_all + SLOTS);
    T.failed = T.tmem_slot + 1;
    const uint32_t tid = threadIdx.x;
    const uint4* s = reinterpret_cast<const uint4*>(w_img);
    uint4* d = reinterpret_cast<uint4*>(smem);
    for (uint32_t i = tid; i < w_bytes / 16; i += 128u * SLOTS) d[i] = s[i];
    if (tid == 0) {
        for (int k = 0; k < SLOTS; ++k)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((uint32_t)__cvta_generic_to_shared(T.mbar_all + k)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        for (int k = 0; k < SLOTS; ++k) T.failed[k] = 0u;
    }
    if ((tid >> 5) == 0) {
        const uint32_t sa = (uint32_t)__cvta_generic_to_shared(T.tmem_slot);
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sa), "r"(64u * SLOTS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    return T;
}

template <int SLOTS>
__device__ __forceinline__ void tc_teardown(const TcTile& T, uint32_t* status) {
    tc_fence_before();
    __syncthreads();
    if ((threadIdx.x >> 5) == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*T.tmem_slot), "r"(64u * SLOTS));
    if (threadIdx.x == 0) {
        uint32_t f = 0;
        for (int k = 0; k < SLOTS; ++k) f |= T.failed[k];
        if (f) atomicOr(status, kStatusTimeout);
    }
}

// one layer of a slot: K / 16 MMAs by the slot's thread 0, committed to the slot's mbarrier, then a
// bounded wait; false when the wait ran out (after the drain wait)
// `between` runs on every thread of the slot after the MMAs are issued and before they are waited
// for (the operand is stable then: written before the first barrier, rewritten after the second)
template <typename F>
__device__ __forceinline__ bool tc_layer(uint32_t r, uint32_t tmem, uint32_t a_addr, uint32_t b_addr, uint32_t K,
                                         uint32_t N, uint32_t mbar_addr, uint32_t& phase, uint32_t slot,
                                         volatile uint32_t* failed, uint32_t max_tries, int issue_mma, F&& between) {
    fence_async_smem();
    tc_fence_before();
    asm volatile("bar.sync %0, 128;" ::"r"(1u + slot) : "memory");
    tc_fence_after();
    if (r == 0 && issue_mma) {
        const uint32_t idesc = umma_idesc(N);
        for (uint32_t j = 0; j < K / 16; ++j)
            umma_bf16(tmem, umma_smem_desc(a_addr + 256u * j, (K / 8) * 128u), umma_smem_desc(b_addr + 256u * j, (K / 8) * 128u),
                      idesc, j > 0 ? 1u : 0u);
        umma_commit(mbar_addr);
    }
    between();
    if (!mbar_wait(mbar_addr, phase, max_tries)) failed[slot] = 1u;
    // every store but the newest (issued by `between`) has read its operand: the buffer this
    // layer's result is written into is free
    if (r == 0) asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
    asm volatile("bar.sync %0, 128;" ::"r"(1u + slot) : "memory");
    if (failed[slot]) {
        if (issue_mma) mbar_wait(mbar_addr, phase, max_tries);
        return false;
    }
    phase ^= 1u;
    tc_fence_after();
    return true;
}

constexpr uint32_t kBwdBuf = (uint32_t)kTcRows * kWidth * 2;  // one A operand: 128 x 64 bf16
constexpr int kBwdSlots = 4;
constexpr int kBwdThreads = 128 * kBwdSlots;
constexpr size_t kBwdTcSmem = 1024 + kUmmaWbBytes + (size_t)kBwdSlots * 2 * kBwdBuf + 128;

// Four slots of 128 records, each with two operand buffers: layer l's A operand (delta_{l+1}, the
// output gradient for l = 5) is buffer l % 2, and delta_l is written into the other one, so that
// the TMA store of one layer's deltas runs on while the next layer's are computed. Each layer's
// mask row h_l is loaded into registers before the layer's MMAs are waited for; the accumulator is
// read 32 columns at a time.
__global__ void __launch_bounds__(kBwdThreads, 1) k_train_bwd_tc(const unsigned char* __restrict__ wb_img,
                                                                 const uint32_t* __restrict__ n_dev, size_t n_max,
                                                                 const __nv_bfloat16* __restrict__ act,
                                                                 const __nv_bfloat16* __restrict__ gout,
                                                                 uint32_t* __restrict__ status, uint32_t max_tries,
                                                                 int issue_mma,
                                                                 const __grid_constant__ CUtensorMap tm_delta_store) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const TcTile T = tc_setup<kBwdSlots>(smem, kUmmaWbBytes, 2 * kBwdBuf, wb_img);
    grid_dependency_wait();  // the forward's activations and output gradients
    launch_dependents();
    const size_t n = n_dev ? min((size_t)*n_dev, n_max) : n_max;
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    const uint32_t slot = tid >> 7, r = tid & 127u;
    unsigned char* bufs = smem + kUmmaWbBytes + slot * 2 * kBwdBuf;
    const uint32_t tmem = *T.tmem_slot + 64u * slot;
    const uint32_t taddr = tmem + ((32u * (warp & 3u)) << 16);
    const uint32_t mbar_addr = (uint32_t)__cvta_generic_to_shared(T.mbar_all + slot);
    const uint32_t sw_addr = (uint32_t)__cvta_generic_to_shared(smem);
    const uint32_t bufs_addr = (uint32_t)__cvta_generic_to_shared(bufs);
    const size_t rows_pad = act_rows(n_max);
    uint32_t phase = 0;
    const size_t n_tiles = (n + kTcRows - 1) / kTcRows;
    bool ok = true;
    for (size_t tile = (size_t)blockIdx.x * kBwdSlots + slot; ok && tile < n_tiles; tile += (size_t)gridDim.x * kBwdSlots) {
        const size_t row = tile * kTcRows + r;
        const bool live = row < n;
        const int g0 = (int)(tile * (kTcRows / 8));  // the tile's first 8-row group
        // the output gradient (48 wide) as the first A operand, in buffer 1
        {
            const uint4* src = reinterpret_cast<const uint4*>(gout + row * kOut);
            unsigned char* dst = bufs + kBwdBuf + (r >> 3) * (kOut / 8) * 128u + (r & 7u) * 16u;
#pragma unroll
            for (int c = 0; c < kOut / 8; ++c)
                *reinterpret_cast<uint4*>(dst + c * 128u) = live ? src[c] : make_uint4(0u, 0u, 0u, 0u);
        }
        for (int l = kLayers - 1; l >= 1 && ok; --l) {
            const uint32_t a_off = (uint32_t)(l & 1) * kBwdBuf;  // this layer's operand; delta_l goes to the other
            // h_l (the mask) on its way while the layer's MMAs run
            uint4 h[kWidth / 8];
            const uint4* hp = reinterpret_cast<const uint4*>(act + (size_t)(l - 1) * rows_pad * kWidth + row * kWidth);
#pragma unroll
            for (int c = 0; c < kWidth / 8; ++c) h[c] = live ? hp[c] : make_uint4(0u, 0u, 0u, 0u);
            // the operand holds delta_{l+1} (l < 5): it leaves by one TMA store while the layer's
            // MMAs read it (rows past the record count are zeros, their masks being zero; whole
            // 8-row groups up to act_rows(n_max))
            ok = tc_layer(r, tmem, bufs_addr + a_off, sw_addr + umma_wb_offset(l), (uint32_t)layer_n(l), (uint32_t)kWidth,
                          mbar_addr, phase, slot, T.failed, max_tries, issue_mma, [&]() {
                              if (l < kLayers - 1 && r == 0) tma_store_5d(&tm_delta_store, 0, 0, 0, g0, l, bufs_addr + a_off);
                          });
            if (!ok) break;
            // mask by h_l > 0 (the ReLU of layer l - 1's output): delta_l, the next A operand
            unsigned char* dst = bufs + (kBwdBuf - a_off) + (r >> 3) * (kWidth / 8) * 128u + (r & 7u) * 16u;
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                float v[32];
                tmem_ld_32x32b<32>(taddr + 32u * half, v);
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const uint4 hh = h[4 * half + c];
                    const uint32_t hw[4] = {hh.x, hh.y, hh.z, hh.w};
                    uint32_t o[4];
                    // h_l is a ReLU output (a zero or positive), so h > 0 is "its 15 magnitude bits
                    // are not zero": the bf16 pair of the accumulator masked by a per-half compare
                    // (the same bits as converting the selected values, a masked half being +0)
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                        o[e] = pack_bf16(v[8 * c + 2 * e], v[8 * c + 2 * e + 1]) & __vcmpne2(hw[e] & 0x7fff7fffu, 0u);
                    *reinterpret_cast<uint4*>(dst + (4 * half + c) * 128u) = make_uint4(o[0], o[1], o[2], o[3]);
                }
            }
        }
        if (ok) {
            // delta_1 (in buffer 0) leaves once every thread has written its row; every store of
            // the tile has read its operand before the next tile writes the buffers
            fence_async_smem();
            asm volatile("bar.sync %0, 128;" ::"r"(1u + slot) : "memory");
            if (r == 0) {
                tma_store_5d(&tm_delta_store, 0, 0, 0, g0, 0, bufs_addr);
                bulk_wait_read();
            }
            asm volatile("bar.sync %0, 128;" ::"r"(1u + slot) : "memory");
        }
    }
    if (r == 0) bulk_wait_all();  // the delta stores are complete before the grid ends
    tc_teardown<kBwdSlots>(T, status);
}

// weight gradients: shared-memory plan of one CTA (bytes from the 1024-aligned base): three
// buffers of one 32-record stage each, so that the loads and encodings of the next two stages
// overlap a stage's MMAs
constexpr int kDwRecords = 32;                                 // records per stage (the UMMA K of a stage)
constexpr uint32_t kDwGroup = (uint32_t)kDwRecords * 16u;      // 8 features of the stage's records: 512 B
constexpr uint32_t kDwA = 16u * kDwGroup;                      // an M = 128 A operand: 128 features x 32 records
constexpr uint32_t kDwLayer = 8u * kDwGroup;                   // 64 features (or outputs) x 32 records: 4 KB
// a buffer: A0 = the encodings (two 128-feature blocks); H = h_1..h_5 back to back; D = delta_1..
// delta_5 back to back; G = the output gradient (6 groups). W_l's A operand (l >= 1) is the M = 128
// window starting at h_l: its upper 64 rows read the next 4 KB (h_{l+1}, or delta_1 after h_5),
// whose products land in accumulator rows 64..127, which are never read.
constexpr uint32_t kDwOffA0 = 0, kDwOffH = 2 * kDwA, kDwOffD = kDwOffH + 5 * kDwLayer, kDwOffG = kDwOffD + 5 * kDwLayer;
constexpr uint32_t kDwBuf = 60u * 1024u;                       // 59 KB used, rounded to 1 KB
static_assert(kDwOffG + 6 * kDwGroup <= kDwBuf, "weight-gradient buffer overflow");
__host__ __device__ constexpr uint32_t dw_off_a(int l) { return kDwOffH + (uint32_t)(l - 1) * kDwLayer; }
// the B operand of W_l: delta_{l+1} (W0..W4), the output gradient (W5)
__host__ __device__ constexpr uint32_t dw_off_b(int l) { return l < 5 ? kDwOffD + (uint32_t)l * kDwLayer : kDwOffG; }
constexpr int kDwBufs = 3;
constexpr uint32_t kDwOffBar = kDwBufs * kDwBuf;               // 180 KB
constexpr size_t kDwTcSmem = 1024 + kDwOffBar + 128;
constexpr int kDwEncWarps = 9;                                 // warp p encodes input p of the stage's 32 records
constexpr int kDwThreads = 32 * (kDwEncWarps + 1);             // + the load/MMA warp
constexpr uint32_t kDwTmemCols = 512;  // dW0 (two M blocks), dW1..dW4, dW5: 7 x 64 columns
// bytes one stage's three TMA loads bring: h_1..h_5, delta_1..delta_5, the output gradient
constexpr uint32_t kDwStageTx = (5u * 8u + 5u * 8u + 6u) * kDwGroup;
// The weight-gradient operands are MN-major (the records, the UMMA K, are the rows of the stored
// activations, the features or outputs contiguous in each): core matrix = 8 records x 8 features
// (16 B per record, 128 B per core matrix); K-adjacent core matrices 128 B apart (leading byte
// offset), MN-adjacent ones 512 B apart (stride byte offset, the 4 record groups of a stage). The 8
// features of group g for all 32 records are therefore one contiguous 512-byte block at g * 512,
// record k at k * 16. This interleaved layout is kept for the output gradient (48 wide, the B
// operand of W5), loaded as a TMA box {8 features, 32 records, 6 groups} (the group dimension's
// stride 16 B, the record's 96 B); the other operands use the 128-byte swizzle below.
constexpr uint32_t kDwLbo = 128u, kDwSbo = (uint32_t)(kDwRecords / 8) * 128u;
// MN-major shared-memory descriptor (no swizzle): leading byte offset = the K stride, stride byte
// offset = the MN stride
// MN-major with the 128-byte swizzle (the layout a TMA box of 64 features x 32 records writes with
// CU_TENSOR_MAP_SWIZZLE_128B): rows of 64 features (128 B, 16-byte chunks XOR-permuted by the row's
// index within its 8-row group), 8 records per 1024-byte group; leading byte offset = the stride
// between 64-feature atoms along MN (4 KB: 32 records), stride byte offset = the 8-record stride
// (1 KB); layout type 2 (128B) in bits 61-63
constexpr uint32_t kDwSwAtom = 4096u, kDwSwGroup = 1024u;
__device__ __forceinline__ uint64_t umma_desc_mn_sw128(uint32_t smem_addr) {
    return (uint64_t)((smem_addr >> 4) & 0x3FFFu) | ((uint64_t)(kDwSwAtom >> 4) << 16) |
           ((uint64_t)(kDwSwGroup >> 4) << 32) | (1ull << 46) | (2ull << 61);
}
__device__ __forceinline__ uint64_t umma_desc_mn(uint32_t smem_addr) {
    return (uint64_t)((smem_addr >> 4) & 0x3FFFu) | ((uint64_t)(kDwLbo >> 4) << 16) |
           ((uint64_t)((kDwSbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// kind::f16 with both operands MN-major (bits 15 and 16)
__host__ __device__ constexpr uint32_t umma_idesc_mn(uint32_t n) { return umma_idesc(n) | (1u << 15) | (1u << 16); }

// mbar_wait that also gives up once another thread of the CTA has marked it failed
__device__ __forceinline__ bool mbar_wait_or_fail(uint32_t addr, uint32_t phase, uint32_t max_tries,
                                                  volatile uint32_t* failed) {
    for (uint32_t i = 0; i < max_tries; i += 256u) {
        if (mbar_wait(addr, phase, 256u)) return true;
        if (*failed) return false;
    }
    return false;
}

// Per CTA a contiguous run of whole 32-record stages, three buffers. Warp 9 (one thread) loads each
// stage's h_1..h_5, delta_1..delta_5 and output gradient by TMA straight into the MN-major operand
// layout (three loads per stage) and issues the stage's 14 MMAs with one commit; warps 0..8 write the stage's layer-0 encodings (warp p: input p of the 32 records; warp 8
// also the raw inputs and the zero padding). Per buffer three mbarriers: tma_full (the loads
// landed), enc_full (the 9 encoder warps arrived), empty (the stage's MMAs completed, so the buffer
// may be refilled). The CTA accumulates all six weight gradients of its records in tensor memory
// (448 of 512 columns; the 64-feature layers use the lower half of M = 128, the upper half zero)
// and writes them as its partial sums. Rows past the record count read as zero: the forward and
// the backward write zero rows up to the end of their last tile, and the TMA fills rows past the
// buffers' extent with zeros.
__global__ void __launch_bounds__(kDwThreads, 1) k_train_dw_tc(
    const __grid_constant__ CUtensorMap tm_act, const __grid_constant__ CUtensorMap tm_delta,
    const __grid_constant__ CUtensorMap tm_gout, const float* __restrict__ rec, const uint32_t* __restrict__ n_dev,
    size_t n_max, Box box, float* __restrict__ part, size_t per_cta, uint32_t* __restrict__ status, uint32_t max_tries,
    int issue_mma) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + kDwOffBar + 3 * kDwBufs * 8);
    volatile uint32_t* failed = tmem_slot + 1;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    const size_t n = n_dev ? min((size_t)*n_dev, n_max) : n_max;
    const size_t c0 = (size_t)blockIdx.x * per_cta, c1 = min(n, c0 + per_cta);
    const int S = c1 > c0 ? (int)((c1 - c0 + kDwRecords - 1) / kDwRecords) : 0;
    const uint32_t base = (uint32_t)__cvta_generic_to_shared(smem);
    // kind 0: tma_full, 1: enc_full, 2: empty
    auto bar = [&](int kind, int b) { return base + kDwOffBar + 8u * (uint32_t)(kDwBufs * kind + b); };
    if (tid == 0) {
        for (int b = 0; b < kDwBufs; ++b) {
            mbar_init(bar(0, b), 1);
            mbar_init(bar(1, b), kDwEncWarps);
            mbar_init(bar(2, b), 1);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        *failed = 0u;
    }
    if (warp == 0) {
        const uint32_t sa = (uint32_t)__cvta_generic_to_shared(tmem_slot);
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sa), "r"(kDwTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    grid_dependency_wait();  // the backward's deltas (and, before it, the forward's activations)
    launch_dependents();
    const uint32_t tmem = *tmem_slot;
    if (warp == (uint32_t)kDwEncWarps) {
        if (lane == 0) {
            // the TMA loads of stage s into buffer s % 3
            auto load_stage = [&](int s) {
                const int b = s % kDwBufs;
                const uint32_t buf = base + (uint32_t)b * kDwBuf, fb = bar(0, b);
                const int y = (int)(c0 + (size_t)s * kDwRecords);
                mbar_arrive_expect_tx(fb, kDwStageTx);
                tma_load_3d(buf + kDwOffH, &tm_act, 0, y, 0, fb);
                tma_load_3d(buf + kDwOffD, &tm_delta, 0, y, 0, fb);
                tma_load_3d(buf + kDwOffG, &tm_gout, 0, y, 0, fb);
            };
            // A and B swizzled (128B), except the output gradient (B of W5), interleaved; a K step of
            // 16 records is two 8-record groups: 2 KB swizzled, 256 B interleaved
            auto issue = [&](uint32_t d_col, uint32_t a, uint32_t bb, uint32_t N, bool acc0, bool b_sw) {
                const uint32_t idesc = umma_idesc_mn(N);
                for (uint32_t j = 0; j < (uint32_t)kDwRecords / 16; ++j)
                    umma_bf16(tmem + d_col, umma_desc_mn_sw128(a + 2u * kDwSwGroup * j),
                              b_sw ? umma_desc_mn_sw128(bb + 2u * kDwSwGroup * j) : umma_desc_mn(bb + 2u * kDwLbo * j), idesc,
                              (acc0 || j > 0) ? 1u : 0u);
            };
            int loaded = 0, landed = 0, committed = 0;  // stages whose loads were issued / waited for / MMAs committed
            if (issue_mma)  // the timeout test issues nothing, so that the first wait runs out
                for (; loaded < min(S, kDwBufs); ++loaded) load_stage(loaded);
            for (int s = 0; s < S; ++s) {
                const int b = s % kDwBufs;
                const uint32_t par = (uint32_t)(s / kDwBufs) & 1u;
                if (!mbar_wait_or_fail(bar(0, b), par, max_tries, failed)) {
                    *failed = 1u;
                    break;
                }
                landed = s + 1;
                if (!mbar_wait_or_fail(bar(1, b), par, max_tries, failed)) {
                    *failed = 1u;
                    break;
                }
                tc_fence_after();
                const uint32_t buf = base + (uint32_t)b * kDwBuf;
                const bool acc = s > 0;
                issue(0u, buf + kDwOffA0, buf + dw_off_b(0), 64u, acc, true);
                issue(64u, buf + kDwOffA0 + kDwA, buf + dw_off_b(0), 64u, acc, true);
                for (int l = 1; l <= 5; ++l)
                    issue(128u + 64u * (uint32_t)(l - 1), buf + dw_off_a(l), buf + dw_off_b(l), (uint32_t)layer_n(l), acc, l < 5);
                umma_commit(bar(2, b));
                committed = s + 1;
                if (s >= 1 && s - 1 + kDwBufs < S) {
                    // refill stage s - 1's buffer with stage s + 2 once stage s - 1's MMAs are done
                    if (!mbar_wait_or_fail(bar(2, (s - 1) % kDwBufs), (uint32_t)((s - 1) / kDwBufs) & 1u, max_tries, failed)) {
                        *failed = 1u;
                        break;
                    }
                    load_stage(s - 1 + kDwBufs);
                    loaded = s - 1 + kDwBufs + 1;
                }
            }
            // every MMA done (the last commit follows all of them); after a failure, also every
            // load still in flight, so that nothing writes this CTA's memory once it has left
            if (!*failed) {
                if (committed > 0 && !mbar_wait_or_fail(bar(2, (committed - 1) % kDwBufs),
                                                        (uint32_t)((committed - 1) / kDwBufs) & 1u, max_tries, failed))
                    *failed = 1u;
            }
            if (*failed) {
                for (int s = landed; s < loaded; ++s) mbar_wait(bar(0, s % kDwBufs), (uint32_t)(s / kDwBufs) & 1u, max_tries);
                if (committed > 0)
                    mbar_wait(bar(2, (committed - 1) % kDwBufs), (uint32_t)((committed - 1) / kDwBufs) & 1u, max_tries);
            }
        }
    } else {
        // encoder warp p: input p of record `lane` of each stage into the stage buffer's A0 (column
        // groups 3p .. 3p + 2); warp 8 also the raw inputs (groups 27, 28) and the zero padding
        const int p = (int)warp;
        float xr[kIn];  // raw inputs of the next stage's record (only those this warp needs)
        auto load_x = [&](int s) {
            const size_t row = c0 + (size_t)s * kDwRecords + lane;
            const bool live = s < S && row < c1;
#pragma unroll
            for (int c = 0; c < kIn; ++c) xr[c] = (live && (p == kIn - 1 || c == p)) ? rec[row * kRecordFloats + c] : 0.0f;
        };
        load_x(0);
        for (int s = 0; s < S; ++s) {
            const int b = s % kDwBufs;
            // the buffer's previous stage (s - 3) has been consumed by its MMAs
            if (s >= kDwBufs && !mbar_wait_or_fail(bar(2, b), (uint32_t)(s / kDwBufs - 1) & 1u, max_tries, failed)) {
                *failed = 1u;
                break;
            }
            const bool live = c0 + (size_t)s * kDwRecords + lane < c1;
            float x[kIn];
            if (live) normalise_input(xr, box.lo, box.inv_ext, x);
            else
                for (int c = 0; c < kIn; ++c) x[c] = 0.0f;
            load_x(s + 1);
            unsigned char* a0 = smem + (uint32_t)b * kDwBuf + kDwOffA0;
            auto put = [&](int g, uint4 v) {
                const uint32_t r8 = lane & 7u;
                *reinterpret_cast<uint4*>(a0 + (uint32_t)(g >> 3) * kDwSwAtom + (lane >> 3) * kDwSwGroup + r8 * 128u +
                                          (((uint32_t)(g & 7) ^ r8) << 4)) = v;
            };
            uint32_t w[kFreq];
            if (live) encode_input(x[p], w);
            else
                for (int k = 0; k < kFreq; ++k) w[k] = 0u;
#pragma unroll
            for (int q = 0; q < 3; ++q) put(3 * p + q, make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]));
            if (p == kIn - 1) {
                put(27, make_uint4(pack_bf16(x[0], x[1]), pack_bf16(x[2], x[3]), pack_bf16(x[4], x[5]), pack_bf16(x[6], x[7])));
                put(28, make_uint4(pack_bf16(x[8], 0.0f), 0u, 0u, 0u));
                for (int g = 29; g < kEnc / 8; ++g) put(g, make_uint4(0u, 0u, 0u, 0u));
            }
            fence_async_smem();  // the generic-proxy stores, visible to the tensor core
            __syncwarp();
            if (lane == 0) mbar_arrive(bar(1, b));
        }
    }
    __syncthreads();
    tc_fence_after();
    // the CTA's partial sums of all six weight gradients to its own slice of part (every entry
    // written, zero when it had no records or gave up), in the parameters' layout; k_adam_reduce
    // adds the slices. Warp w < 8 reads lane quarter w % 4 (features 32 (w % 4) ..); warps 0-3 take
    // dW0 and dW1, 4-7 dW2..dW5; a thread's row leaves as float4 stores.
    if (warp < 8) {
        const bool have = !*failed && S > 0 && issue_mma;  // uniform over the CTA
        float* P = part + (size_t)blockIdx.x * kParams;
        const uint32_t q = warp & 3u, m = 32u * q + lane;
        const uint32_t lane_base = (32u * q) << 16;
        for (int acc_i = (warp < 4 ? 0 : 3); acc_i < (warp < 4 ? 3 : 7); ++acc_i) {
            if (acc_i >= 2 && q >= 2) continue;  // dW1..dW5 have 64 features: lane quarters 0 and 1
            float v[64];
            if (have) tmem_ld_x64(tmem + lane_base + 64u * (uint32_t)acc_i, v);
            else
                for (int c = 0; c < 64; ++c) v[c] = 0.0f;
            const int l = acc_i <= 1 ? 0 : acc_i - 1, N = layer_n(l);
            const uint32_t row = acc_i <= 1 ? m + 128u * (uint32_t)acc_i : m;  // dW0: block 1 holds features 128..255
            float4* G = reinterpret_cast<float4*>(P + param_offset(l) + (size_t)row * N);
#pragma unroll
            for (int c = 0; c < 16; ++c)
                if (4 * c < N) G[c] = make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kDwTmemCols));
    if (tid == 0 && *failed) atomicOr(status, kStatusTimeout);
}

// The weight gradient (the sum of the nparts partial slices of k_train_dw_tc, in a fixed order, so
// that a step is reproducible) and Adam on the f32 master weights, each new weight also packed
// into the bf16 operand images. A block covers 32 float4
// columns of parameters; its 32 warps sum every 32nd slice each (at most 5 loads, all in flight
// together), then warp 0 adds the 32 sums.
constexpr int kReduceCols = 32, kReduceGroups = 32, kReduceMaxParts = 160;
__global__ void __launch_bounds__(kReduceCols * kReduceGroups) k_adam_reduce(
    const float* __restrict__ part, int nparts, float* __restrict__ P, float* __restrict__ M, float* __restrict__ V,
    float t, float lr, float b1, float b2, float eps, float* __restrict__ grad_out, unsigned char* __restrict__ img,
    unsigned char* __restrict__ img_b) {
    __shared__ float4 sums[kReduceGroups][kReduceCols];
    grid_dependency_wait();  // the weight-gradient partial sums
    launch_dependents();
    const int lane = threadIdx.x % kReduceCols, grp = threadIdx.x / kReduceCols;
    const int c4 = blockIdx.x * kReduceCols + lane;
    const bool live = c4 < kParams / 4;
    float4 acc = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (live) {
        float4 x[kReduceMaxParts / kReduceGroups];
#pragma unroll
        for (int k = 0; k < kReduceMaxParts / kReduceGroups; ++k) {
            const int p = grp + k * kReduceGroups;
            x[k] = p < nparts ? __ldcs(reinterpret_cast<const float4*>(part + (size_t)p * kParams) + c4)
                              : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
#pragma unroll
        for (int k = 0; k < kReduceMaxParts / kReduceGroups; ++k) {
            acc.x += x[k].x;
            acc.y += x[k].y;
            acc.z += x[k].z;
            acc.w += x[k].w;
        }
    }
    sums[grp][lane] = acc;
    __syncthreads();
    if (grp != 0 || !live) return;
    float g[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int k = 0; k < kReduceGroups; ++k) {
        g[0] += sums[k][lane].x;
        g[1] += sums[k][lane].y;
        g[2] += sums[k][lane].z;
        g[3] += sums[k][lane].w;
    }
    if (grad_out) reinterpret_cast<float4*>(grad_out)[c4] = make_float4(g[0], g[1], g[2], g[3]);
    if (lr <= 0.0f) return;  // gradients only
    const float c1 = 1.0f - powf(b1, t), c2 = 1.0f - powf(b2, t);  // t: the step being taken, from 1
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int i = 4 * c4 + j;
        const float m = b1 * M[i] + (1.0f - b1) * g[j];
        const float v = b2 * V[i] + (1.0f - b2) * g[j] * g[j];
        M[i] = m;
        V[i] = v;
        const float mh = m / c1, vh = v / c2;
        const float p = P[i] - lr * mh / (sqrtf(vh) + eps);
        P[i] = p;
        pack_param(i, p, img, img_b);  // the new weight into both bf16 operand images
    }
}

// launches kernel with programmatic stream serialization (grid_dependency_wait): its CTAs may
// start, and run the part before their wait, while the previous kernel of the stream finishes
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t st,
                       Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

int launch_pack(liar_gpu_guide* G, cudaStream_t st) {
    k_pack_umma<<<(kParams + 255) / 256, 256, 0, st>>>(G->params, G->umma_w, G->umma_wb);
    return cudaGetLastError() == cudaSuccess ? LIAR_OK : LIAR_ERR_CUDA;
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
    void* p = nullptr;
    if (G->part_cap < ctx->num_sms) {
        if (G->grad_part) {
            cudaFree(G->grad_part);
            G->buffers.erase(std::remove(G->buffers.begin(), G->buffers.end(), (void*)G->grad_part), G->buffers.end());
        }
        G->grad_part = nullptr;
        G->part_cap = 0;
        int rc = g_alloc(ctx, G, (size_t)ctx->num_sms * kParams * sizeof(float), &p, "guide gradient partial sums");
        if (rc) return rc;
        G->grad_part = static_cast<float*>(p);
        G->part_cap = ctx->num_sms;
    }
    if (!G->wpart) {
        int rc = g_alloc(ctx, G, kWeightParts * sizeof(float), &p, "guide weight sums");
        if (rc) return rc;
        G->wpart = static_cast<float*>(p);
    }
    if (G->cap >= n) return LIAR_OK;
    for (void* q : {(void*)G->act, (void*)G->delta, (void*)G->gout}) {
        if (!q) continue;
        cudaFree(q);
        G->buffers.erase(std::remove(G->buffers.begin(), G->buffers.end(), q), G->buffers.end());
    }
    G->act = G->delta = G->gout = nullptr;
    G->cap = 0;
    int rc = g_alloc(ctx, G, act_rows(n) * 5 * kWidth * 2, &p, "guide activations");
    if (rc) return rc;
    G->act = static_cast<__nv_bfloat16*>(p);
    rc = g_alloc(ctx, G, act_rows(n) * 5 * kWidth * 2, &p, "guide deltas");
    if (rc) return rc;
    G->delta = static_cast<__nv_bfloat16*>(p);
    rc = g_alloc(ctx, G, n * kOut * 2, &p, "guide output gradients");
    if (rc) return rc;
    G->gout = static_cast<__nv_bfloat16*>(p);
    // rows past a step's record count are read as zero operands; start them at zero
    cudaError_t e = cudaMemset(G->act, 0, act_rows(n) * 5 * kWidth * 2);
    if (e == cudaSuccess) e = cudaMemset(G->delta, 0, act_rows(n) * 5 * kWidth * 2);
    if (e == cudaSuccess) e = cudaMemset(G->gout, 0, n * kOut * 2);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "guide training buffers");
    G->tm_base = nullptr;
    G->cap = n;
    return LIAR_OK;
}

// cuTensorMapEncodeTiled from the driver, through the runtime (the library links no driver stub)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
        else
            cudaGetLastError();
    }
    return fn;
}

// The weight-gradient kernel's TMA descriptors for n_max records: act and delta ([5][n_max][64]
// bf16) as 3D tensors {64 features, n_max records, 5 layers}, boxes {64, 32, 5} with the 128-byte
// swizzle (the MN-major swizzled operand layout, five layers back to back); the output gradient
// ([n_max][48]) as {8 features, n_max records (stride 96 B), 6 groups (stride 16 B)}, boxes
// {8, 32, 6}, unswizzled (the interleaved MN-major layout). Rows past n_max read as zero.
// Re-encoded when the buffers or the record count change.
int ensure_tensor_maps(liar_gpu_ctx* ctx, liar_gpu_guide* G, size_t n_max) {
    if (G->tm_base == G->act && G->tm_rows == n_max) return LIAR_OK;
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return ctx_fail(ctx, LIAR_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const cuuint32_t box4[3] = {(cuuint32_t)kWidth, (cuuint32_t)kDwRecords, 5}, box3[3] = {8, (cuuint32_t)kDwRecords, 6};
    const cuuint32_t unit[4] = {1, 1, 1, 1};
    const cuuint64_t dims4[3] = {(cuuint64_t)kWidth, (cuuint64_t)n_max, 5};
    const cuuint64_t strides4[2] = {(cuuint64_t)kWidth * 2, (cuuint64_t)act_rows(n_max) * kWidth * 2};
    const cuuint64_t dims3[3] = {8, (cuuint64_t)n_max, 6};
    const cuuint64_t strides3[2] = {(cuuint64_t)kOut * 2, 16};
    CUresult r = enc(&G->tm_act, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, G->act, dims4, strides4, box4, unit,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r == CUDA_SUCCESS)
        r = enc(&G->tm_delta, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, G->delta, dims4, strides4, box4, unit,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r == CUDA_SUCCESS)
        r = enc(&G->tm_gout, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, G->gout, dims3, strides3, box3, unit,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    // the tile stores: {8 features, 8 rows (stride 128 B), 8 chunks (stride 16 B), row groups
    // (stride 1 KB), 5 layers}, boxes of one 128-row tile {8, 8, 8, 16, 1} read from the K-major
    // core-matrix layout of a slot's operand (row r, chunk c at (r / 8) * 1024 + c * 128 + (r % 8) * 16)
    const cuuint64_t rows_pad = act_rows(n_max);
    const cuuint64_t dims5[5] = {8, 8, 8, rows_pad / 8, 5};
    const cuuint64_t strides5[4] = {(cuuint64_t)kWidth * 2, 16, 8 * (cuuint64_t)kWidth * 2, rows_pad * kWidth * 2};
    const cuuint32_t box5[5] = {8, 8, 8, (cuuint32_t)kTcRows / 8, 1}, unit5[5] = {1, 1, 1, 1, 1};
    if (r == CUDA_SUCCESS)
        r = enc(&G->tm_act_st, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, G->act, dims5, strides5, box5, unit5,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r == CUDA_SUCCESS)
        r = enc(&G->tm_delta_st, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, G->delta, dims5, strides5, box5, unit5,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        G->tm_base = nullptr;
        return ctx_fail(ctx, LIAR_ERR_CUDA, "TMA descriptor encoding failed (CUresult %d)", (int)r);
    }
    G->tm_base = G->act;
    G->tm_rows = n_max;
    return LIAR_OK;
}

int smem_attrs(liar_gpu_ctx* ctx) {
    static int done_device = -1;
    if (done_device == ctx->device) return LIAR_OK;
    cudaError_t e = cudaFuncSetAttribute(k_train_bwd_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBwdTcSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_train_dw_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDwTcSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_eval_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEvSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_eval_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEvSmem);
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
    const int sms = ctx->num_sms;
    const unsigned wgrid = (unsigned)std::max<size_t>(1, std::min<size_t>((n_max + 255) / 256, (size_t)kWeightParts));
    // launched programmatically as well (it waits for the kernel before it, a previous step's Adam
    // kernel or whatever wrote the records, before reading anything), and it clears the loss sum
    cudaError_t e = launch_pdl(k_weight_sum, wgrid, 256, 0, st, d_records, d_count, n_max, G->wpart, G->scalars + 1);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "guide weight sum");
    // the bounded waits of the tensor-core kernels (the fault test: no MMA, a short limit)
    const bool wait_test = ctx->fault_test == LIAR_FAULT_TEST_GUIDE_WAIT;
    const uint32_t tries = wait_test ? 1u << 16 : 1u << 24;
    const int mma = wait_test ? 0 : 1;
    uint32_t* status = ctx->d_scratch + kStatusWord;
    const size_t tiles = (n_max + kTcRows - 1) / kTcRows;
    // forward: the inference kernel's four slots storing h_1..h_5, the loss and the output
    // gradient per record
    const unsigned tgrid = (unsigned)std::max<size_t>(1, std::min<size_t>((tiles + kEvSlots - 1) / kEvSlots, (size_t)sms));
    rc = ensure_tensor_maps(ctx, G, n_max);
    if (rc) return rc;
    // the kernels after k_weight_sum start programmatically: each one's prologue (weights to shared
    // memory, barriers, tensor memory) overlaps the end of the kernel before it
    e = launch_pdl(k_eval_tc<true>, tgrid, kEvThreads, kEvSmem, st, G->umma_w, d_records, n_max, box, 0,
                   status, tries, mma, d_count, n_max, G->scalars, G->gout, (const float*)G->wpart, (int)wgrid,
                   G->tm_act_st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "guide training forward");
    const unsigned bgrid =
        (unsigned)std::max<size_t>(1, std::min<size_t>((tiles + kBwdSlots - 1) / kBwdSlots, (size_t)sms));
    e = launch_pdl(k_train_bwd_tc, bgrid, kBwdThreads, kBwdTcSmem, st, G->umma_wb, d_count, n_max, G->act, G->gout,
                   status, tries, mma, G->tm_delta_st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "guide training backward");
    // weight gradients: one CTA per SM, each over a contiguous run of whole 32-record stages
    const size_t stages = (n_max + kDwRecords - 1) / kDwRecords;
    const size_t ctas = (size_t)std::min(sms, kReduceMaxParts);  // partial slices k_adam_reduce can add
    const size_t per_cta = ((stages + ctas - 1) / ctas) * kDwRecords;
    const unsigned dgrid = (unsigned)std::max<size_t>(1, (n_max + per_cta - 1) / per_cta);
    e = launch_pdl(k_train_dw_tc, dgrid, kDwThreads, kDwTcSmem, st, G->tm_act, G->tm_delta, G->tm_gout, d_records,
                   d_count, n_max, box, G->grad_part, per_cta, status, tries, mma);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "guide weight gradients");
    const float lr = apply ? (G->cfg.learning_rate > 0 ? G->cfg.learning_rate : 5e-3f) : 0.0f;
    e = launch_pdl(k_adam_reduce, (kParams / 4 + kReduceCols - 1) / kReduceCols, kReduceCols * kReduceGroups, 0, st,
                   G->grad_part, (int)dgrid, G->params, G->adam_m, G->adam_v, (float)(G->steps_done + 1), lr, 0.9f,
                   0.99f, 1e-8f, d_grad_out, G->umma_w, G->umma_wb);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "guide Adam step");
    if (apply) G->steps_done += 1;
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
    rc = g_alloc(ctx, G, 3 * (size_t)kParams * sizeof(float) + 256, &p, "guide parameters");
    if (!rc) {
        float* f = static_cast<float*>(p);
        G->params = f;
        G->adam_m = f + kParams;
        G->adam_v = f + 2 * kParams;
        G->scalars = f + 3 * kParams + 4;  // after 4 spare floats
    }
    if (!rc) rc = g_alloc(ctx, G, kUmmaWBytes, &p, "guide operand images");
    if (!rc) G->umma_w = static_cast<unsigned char*>(p);
    if (!rc) rc = g_alloc(ctx, G, kUmmaWbBytes, &p, "guide operand images");
    if (!rc) G->umma_wb = static_cast<unsigned char*>(p);
    if (!rc) {
        std::vector<float> P;
        init_params(P, cfg->seed);
        cudaError_t e = cudaMemcpy(G->params, P.data(), kParams * sizeof(float), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemset(G->adam_m, 0, 2 * (size_t)kParams * sizeof(float) + 256);
        if (e != cudaSuccess) rc = ctx_cuda(ctx, e, "guide initialisation");
    }
    if (!rc && launch_pack(G, ctx->stream)) rc = ctx_cuda(ctx, cudaGetLastError(), "guide pack");
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
    if (e == cudaSuccess) e = cudaMemset(G->adam_m, 0, 2 * (size_t)kParams * sizeof(float) + 256);  // Adam moments
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "guide parameters");
    if (launch_pack(G, ctx->stream)) return ctx_cuda(ctx, cudaGetLastError(), "guide pack");
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
    if ((uintptr_t)d_mixture & 15u) return ctx_fail(ctx, LIAR_ERR_INVALID, "mixture output not 16-byte aligned");
    const unsigned grid = (unsigned)std::max<size_t>(1, std::min<size_t>((tiles + kEvSlots - 1) / kEvSlots, (size_t)ctx->num_sms));
    // the mixtures leave each slot as one TMA store: a 2D map over [n][stride] floats, boxes of
    // 128 rows (rows past n are not written)
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return ctx_fail(ctx, LIAR_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    CUtensorMap tm_mix;
    const cuuint64_t dims[2] = {(cuuint64_t)stride, (cuuint64_t)n}, strides[1] = {(cuuint64_t)stride * 4};
    const cuuint32_t box[2] = {(cuuint32_t)stride, (cuuint32_t)kTcRows}, unit[2] = {1, 1};
    const CUresult cr = enc(&tm_mix, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, d_mixture, dims, strides, box, unit,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return ctx_fail(ctx, LIAR_ERR_CUDA, "TMA descriptor encoding failed (CUresult %d)", (int)cr);
    // the bounded waits' limit: 2^24 polls, far beyond a layer's MMAs; the timeout test
    // (liar_gpu_set_fault_test) issues no MMA and gives up after 2^16 polls
    const bool wait_test = ctx->fault_test == LIAR_FAULT_TEST_GUIDE_WAIT;
    k_eval_tc<false><<<grid, kEvThreads, kEvSmem, st>>>(G->umma_w, d_inputs, n, make_box(G->cfg), stride,
                                                          ctx->d_scratch + kStatusWord, wait_test ? 1u << 16 : 1u << 24,
                                                          wait_test ? 0 : 1, nullptr, 0, nullptr, nullptr, nullptr, 0,
                                                          tm_mix);
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
