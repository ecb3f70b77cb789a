// guide_mlp.cuh -- the path-guiding network on the tensor cores (no reference counterpart).
//
// Network: 9 inputs (position normalised to the scene box, shading normal, direction to the
// previous vertex) -> frequency encoding (per input: sin and cos of pi * 2^(f/2) * x, f = 0..11, then
// the 9 raw inputs; 225 features, padded to 256) -> 5 ReLU layers of 64 -> 48 outputs (40 used):
// 8 von Mises-Fisher lobes, each (mean direction m 3, log concentration 1, logit 1). No biases.
// Weights are bf16, accumulation f32. Inference and training run on tcgen05 (guide_umma.cuh,
// guide.cu).
//
// Parameters (f32 master copy, row-major [in][out]): W0 256x64, W1..W4 64x64, W5 64x48. For the
// kernels they are packed as bf16 tcgen05 B-operand images, forward and transposed (guide.cu
// pack_param).
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

namespace liar_gpu {
namespace guide {

constexpr int kIn = 9;
constexpr int kFreq = 12;
constexpr int kEncUsed = kIn * 2 * kFreq + kIn;  // 225
constexpr int kEnc = 256;
constexpr int kWidth = 64;
constexpr int kOut = 48;
constexpr int kOutUsed = 40;
constexpr int kLobes = 8;
constexpr int kLayers = 6;  // W0..W5

__host__ __device__ constexpr int layer_k(int l) { return l == 0 ? kEnc : kWidth; }
__host__ __device__ constexpr int layer_n(int l) { return l == 5 ? kOut : kWidth; }
__host__ __device__ constexpr int param_offset(int l) {
    return l == 0 ? 0 : (l <= 5 ? kEnc * kWidth + (l - 1) * kWidth * kWidth : kEnc * kWidth + 4 * kWidth * kWidth + kWidth * kOut);
}
constexpr int kParams = param_offset(6);  // 35840

#ifdef __CUDACC__

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// max(lo, 0) and max(hi, 0) as a bf16 pair in one conversion (cvt.rn.relu: rounded to nearest
// even, negative results clamped to zero); equal to pack_bf16(fmaxf(lo, 0), fmaxf(hi, 0)) for
// every input but NaN
__device__ __forceinline__ uint32_t pack_bf16_relu(float lo, float hi) {
    uint32_t d;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
    return d;
}

__device__ __forceinline__ float bf16_lo(uint32_t v) { return __uint_as_float(v << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t v) { return __uint_as_float(v & 0xffff0000u); }

// The encoding of one row as 256 bf16 in a row-major buffer (encode_row_umma of guide_umma.cuh
// writes the same values into the K-major operand layout). Per input two sincospi_enc calls (pi x and
// pi x sqrt(2)); the other frequencies by the doubling formulas sin 2a = 2 sin a cos a,
// cos 2a = cos^2 a - sin^2 a (x fl(sqrt 2) 2^k is exactly fl(x fl(sqrt 2)) 2^k, so these are the
// angles of the definition; the recurrence adds ~1e-6 absolute error, far below bf16).

// sin(pi x) and cos(pi x) for the encodings (|x| < 2^21): x = n / 2 + r with n the nearest integer
// to 2x (found by adding 1.5 * 2^23, whose low mantissa bits then hold n) and |r| <= 1/4, so that
// r = x - n / 2 is exact; the Taylor polynomials of sin and cos about 0 up to the 11th and 10th
// degree on |pi r| <= pi / 4 (truncation below 2e-9 and 1e-8), then the quarter-turn n mod 4
// rotates (sin, cos). Absolute error a few 1e-8, far below the bf16 rounding of the encodings.
__device__ __forceinline__ void sincospi_enc(float x, float* sp, float* cp) {
    const float t = x + x;
    const float big = t + 12582912.0f;  // 1.5 * 2^23
    const int n = __float_as_int(big) - 0x4B400000;
    const float nf = big - 12582912.0f;
    const float r = fmaf(nf, -0.5f, x);
    const float a = r * 3.14159265358979323846f;
    const float a2 = a * a;
    float ps = fmaf(a2, -2.50521083854417188e-8f, 2.75573192239858907e-6f);  // -1/11!, 1/9!
    ps = fmaf(a2, ps, -1.98412698412698413e-4f);                             // -1/7!
    ps = fmaf(a2, ps, 8.33333333333333333e-3f);                              // 1/5!
    ps = fmaf(a2, ps, -1.66666666666666667e-1f);                             // -1/3!
    const float sn = fmaf(a * a2, ps, a);
    float pc = fmaf(a2, 2.08767569878680990e-9f, -2.75573192239858907e-7f);  // 1/12!, -1/10!
    pc = fmaf(a2, pc, 2.48015873015873016e-5f);                              // 1/8!
    pc = fmaf(a2, pc, -1.38888888888888889e-3f);                             // -1/6!
    pc = fmaf(a2, pc, 4.16666666666666667e-2f);                              // 1/4!
    pc = fmaf(a2, pc, -0.5f);                                                // -1/2!
    const float cs = fmaf(a2, pc, 1.0f);
    const int q = n & 3;
    const float s_ = (q & 1) ? cs : sn, c_ = (q & 1) ? sn : cs;
    *sp = (q & 2) ? -s_ : s_;
    *cp = ((q + 1) & 2) ? -c_ : c_;
}

// packed pairs of f32 (Blackwell's two-wide FP32 instructions): every lane rounds exactly as the
// scalar operation would
__device__ __forceinline__ uint64_t f2_make(float lo, float hi) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void f2_split(uint64_t v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ uint64_t f2_fma(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ uint64_t f2_mul(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t f2_add(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t f2_splat(float a) { return f2_make(a, a); }

// the 12 words (24 bf16: sin/cos pairs of the 12 frequencies) of input value xd, as encode_row:
// the two angle chains (pi x and pi x sqrt 2) run side by side as f32x2 pairs, each lane with the
// operations and roundings of sincospi_enc and the doubling formulas
__device__ __forceinline__ void encode_input(float xd, uint32_t* w) {
    const float x0 = xd, x1 = xd * 1.41421356237309515f;
    // x = n / 2 + r, |r| <= 1/4, as in sincospi_enc (the integer quadrants per lane)
    const float b0 = (x0 + x0) + 12582912.0f, b1 = (x1 + x1) + 12582912.0f;
    const int q0 = (__float_as_int(b0) - 0x4B400000) & 3, q1 = (__float_as_int(b1) - 0x4B400000) & 3;
    const uint64_t X = f2_make(x0, x1);
    const uint64_t NF = f2_make(b0 - 12582912.0f, b1 - 12582912.0f);
    const uint64_t R = f2_fma(NF, f2_splat(-0.5f), X);
    const uint64_t A = f2_mul(R, f2_splat(3.14159265358979323846f));
    const uint64_t A2 = f2_mul(A, A);
    uint64_t ps = f2_fma(A2, f2_splat(-2.50521083854417188e-8f), f2_splat(2.75573192239858907e-6f));
    ps = f2_fma(A2, ps, f2_splat(-1.98412698412698413e-4f));
    ps = f2_fma(A2, ps, f2_splat(8.33333333333333333e-3f));
    ps = f2_fma(A2, ps, f2_splat(-1.66666666666666667e-1f));
    const uint64_t SN = f2_fma(f2_mul(A, A2), ps, A);
    uint64_t pc = f2_fma(A2, f2_splat(2.08767569878680990e-9f), f2_splat(-2.75573192239858907e-7f));
    pc = f2_fma(A2, pc, f2_splat(2.48015873015873016e-5f));
    pc = f2_fma(A2, pc, f2_splat(-1.38888888888888889e-3f));
    pc = f2_fma(A2, pc, f2_splat(4.16666666666666667e-2f));
    pc = f2_fma(A2, pc, f2_splat(-0.5f));
    const uint64_t CS = f2_fma(A2, pc, f2_splat(1.0f));
    float sn0, sn1, cs0, cs1;
    f2_split(SN, sn0, sn1);
    f2_split(CS, cs0, cs1);
    // the quarter-turn n mod 4 of each lane
    const float t0 = (q0 & 1) ? cs0 : sn0, u0 = (q0 & 1) ? sn0 : cs0;
    const float t1 = (q1 & 1) ? cs1 : sn1, u1 = (q1 & 1) ? sn1 : cs1;
    uint64_t S = f2_make((q0 & 2) ? -t0 : t0, (q1 & 2) ? -t1 : t1);
    uint64_t C = f2_make(((q0 + 1) & 2) ? -u0 : u0, ((q1 + 1) & 2) ? -u1 : u1);
#pragma unroll
    for (int k = 0; k < kFreq / 2; ++k) {
        float s0, s1, c0, c1;
        f2_split(S, s0, s1);
        f2_split(C, c0, c1);
        w[2 * k] = pack_bf16(s0, c0);
        w[2 * k + 1] = pack_bf16(s1, c1);
        // sin 2a = (2 sin a) cos a, cos 2a = cos a cos a - sin a sin a
        const uint64_t NS = f2_mul(f2_add(S, S), C);
        const uint64_t SS = f2_mul(S, S);
        float ss0, ss1;
        f2_split(SS, ss0, ss1);
        C = f2_fma(C, C, f2_make(-ss0, -ss1));
        S = NS;
    }
}

__device__ __forceinline__ void encode_row(const float* x, __nv_bfloat16* row) {
    uint32_t* dst = reinterpret_cast<uint32_t*>(row);
#pragma unroll
    for (int d = 0; d < kIn; ++d) {
        float s0, c0, s1, c1;
        sincospi_enc(x[d], &s0, &c0);
        sincospi_enc(x[d] * 1.41421356237309515f, &s1, &c1);
        uint32_t* w = dst + d * kFreq;  // pair index (d * 24 + 2 f) / 2
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
    }
    uint32_t* raw = dst + kIn * kFreq;  // columns 216..255
#pragma unroll
    for (int c = 0; c < 4; ++c) raw[c] = pack_bf16(x[2 * c], x[2 * c + 1]);
    raw[4] = pack_bf16(x[8], 0.0f);
#pragma unroll
    for (int c = 5; c < (kEnc - kIn * 2 * kFreq) / 2; ++c) raw[c] = 0u;
}

#endif  // __CUDACC__

// ---- the mixture (host and device)

#ifdef __CUDACC__
#define GM_HD __host__ __device__ __forceinline__
#else
#define GM_HD inline
#endif

// concentration exp(clamp(s)); the mean's gradient uses 1 / max(|m|, kMeanNormMin)
constexpr float kLogKappaMin = -6.0f, kLogKappaMax = 7.0f, kMeanNormMin = 1e-3f;

struct Lobe {
    float mx, my, mz, kappa;
};

// raw outputs (40) -> lobes (unit mean, concentration) and weights (softmax)
GM_HD void mixture_from_raw(const float* o, Lobe* lobes, float* w) {
    float mx = -3.0e38f;
    for (int l = 0; l < kLobes; ++l) mx = fmaxf(mx, o[5 * l + 4]);
    float sum = 0.0f;
    for (int l = 0; l < kLobes; ++l) {
        const float x = o[5 * l], y = o[5 * l + 1], z = o[5 * l + 2];
        const float n = sqrtf(x * x + y * y + z * z);
        if (n > 0.0f) {
            const float inv = 1.0f / n;
            lobes[l].mx = x * inv;
            lobes[l].my = y * inv;
            lobes[l].mz = z * inv;
        } else {
            lobes[l].mx = lobes[l].my = 0.0f;
            lobes[l].mz = 1.0f;
        }
        lobes[l].kappa = expf(fminf(fmaxf(o[5 * l + 3], kLogKappaMin), kLogKappaMax));
        w[l] = expf(o[5 * l + 4] - mx);
        sum += w[l];
    }
    for (int l = 0; l < kLobes; ++l) w[l] /= sum;
}

// log of the vMF density on the unit sphere: kappa / (2 pi (1 - e^{-2 kappa})) e^{kappa (mu.w - 1)}
GM_HD float vmf_log_pdf(float kappa, float cos_t) {
    return logf(kappa / (-expm1f(-2.0f * kappa))) - 1.8378770664093453f /* log 2 pi */ + kappa * (cos_t - 1.0f);
}

// the vMF normalisation kappa / (2 pi (1 - e^{-2 kappa}))
GM_HD float vmf_norm(float kappa) { return kappa / (6.283185307179586f * -expm1f(-2.0f * kappa)); }

// the renderer's copy of a mixture carries each lobe's weight times its normalisation as well
constexpr int kMixRender = 48;

#ifdef __CUDACC__
// ---- the mixture as stored by the network's inference: m[0..31] = 8 x (mu x, y, z, kappa),
// m[32..39] = the 8 weights (and, in the renderer's copy, m[40..47] = weight x vmf_norm(kappa))

// the density from the renderer's copy: one exponential per lobe
__device__ __forceinline__ float mixture_pdf_render(const float* m, float dx, float dy, float dz) {
    float p = 0.0f;
#pragma unroll
    for (int l = 0; l < kLobes; ++l) {
        const float c = m[4 * l] * dx + m[4 * l + 1] * dy + m[4 * l + 2] * dz;
        p += m[40 + l] * expf(m[4 * l + 3] * (c - 1.0f));
    }
    return p;
}

__device__ __forceinline__ float mixture_pdf(const float* m, float dx, float dy, float dz) {
    float p = 0.0f;
#pragma unroll
    for (int l = 0; l < kLobes; ++l) {
        const float c = m[4 * l] * dx + m[4 * l + 1] * dy + m[4 * l + 2] * dz;
        p += m[32 + l] * expf(vmf_log_pdf(m[4 * l + 3], c));
    }
    return p;
}

// lobe by weight (u0), then the vMF's cosine by its inverse CDF, w = 1 + log(u1 + (1 - u1) e^{-2k}) / k
// (Jakob 2012), azimuth 2 pi u2 in the frame of Duff et al. 2017 around the mean
__device__ __forceinline__ void mixture_sample(const float* m, float u0, float u1, float u2, float& dx, float& dy,
                                               float& dz) {
    int lobe = kLobes - 1;
    float acc = 0.0f;
#pragma unroll
    for (int l = 0; l < kLobes; ++l) {
        acc += m[32 + l];
        if (u0 < acc && lobe == kLobes - 1 && l < kLobes - 1) lobe = l;
    }
    // (the first l with u0 < acc; the last lobe takes the rounding remainder)
    float mx = m[0], my = m[1], mz = m[2], k = m[3];
#pragma unroll
    for (int l = 1; l < kLobes; ++l)
        if (l == lobe) {
            mx = m[4 * l];
            my = m[4 * l + 1];
            mz = m[4 * l + 2];
            k = m[4 * l + 3];
        }
    float w = 1.0f + logf(u1 + (1.0f - u1) * expf(-2.0f * k)) / k;
    w = fminf(1.0f, fmaxf(-1.0f, w));
    const float s = sqrtf(fmaxf(0.0f, 1.0f - w * w));
    const float sign = copysignf(1.0f, mz);
    const float a = -1.0f / (sign + mz);
    const float b = mx * my * a;
    const float tx = 1.0f + sign * mx * mx * a, ty = sign * b, tz = -sign * mx;
    const float bx = b, by = sign + my * my * a, bz = -my;
    float sp, cp;
    sincospif(2.0f * u2, &sp, &cp);
    dx = w * mx + s * (cp * tx + sp * bx);
    dy = w * my + s * (cp * ty + sp * by);
    dz = w * mz + s * (cp * tz + sp * bz);
}
#endif

#undef GM_HD

}  // namespace guide
}  // namespace liar_gpu
