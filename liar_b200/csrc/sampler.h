// sampler.h -- the per-pixel stratified sampler of the renderer (host and device).
//
// Plays the role of the reference's Stratifier (src/liar/samplers/stratifier.cpp:163-260): every
// sample dimension of a pixel is stratified over the pixel's spp samples (one jittered stratum
// per sample, strata assigned to samples by a pseudo-random permutation per pixel and
// dimension), and the dimensions of a path generation are the AdjointPhotonTracer's
// sub-sequences (src/liar/tracers/adjoint_photon_tracer.cpp:47-67). Beyond maxRayGeneration the
// reference draws plain random numbers (mt19937); here those dimensions are plain hashes.
//
// Unlike the reference's sequential mt19937 the values are a pure function of (seed, pixel,
// sample, dimension), so any thread can draw any sample in any order:
//   h      = splitmix64 finaliser (Steele, Lea, Flood 2014) of seed and (pixel, dimension)
//   jitter = top 24 bits of splitmix64(h + sample), in [0, 1)
//   stratum= a bijection of [0, spp) keyed by h: a 4-round Feistel network on the next even
//            power of two, cycle-walked into [0, spp) (Black & Rogaway 2002)
//   value  = (stratum + jitter) / spp
// Screen and lens samples are 2D-stratified (sample_2d), as the reference's Stratifier does.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define LS_HD __host__ __device__ __forceinline__
#else
#define LS_HD inline
#endif

namespace liar_gpu {

LS_HD uint64_t mix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

LS_HD float to_unit(uint64_t h) { return (float)(uint32_t)(h >> 40) * (1.0f / 16777216.0f); }

LS_HD uint32_t permute_index(uint32_t i, uint32_t n, uint64_t key) {
    if (n <= 1) return 0;
    uint32_t bits = 0;
    while ((1u << bits) < n) ++bits;
    if (bits & 1u) ++bits;
    const uint32_t half = bits / 2, mask = (1u << half) - 1u;
    do {
        uint32_t l = i >> half, r = i & mask;
        for (uint32_t round = 0; round < 4; ++round) {
            const uint32_t f = (uint32_t)mix64(key + 0x632be59bd9b4e019ull * (round + 1) + r) & mask;
            const uint32_t nl = r;
            r = l ^ f;
            l = nl;
        }
        i = (l << half) | r;
    } while (i >= n);
    return i;
}

// sample dimensions
enum : uint32_t {
    DIM_SCREEN = 0,   // 2 ids
    DIM_LENS = 2,     // 2 ids
    DIM_LAMBDA = 4,
    DIM_GEN0 = 8,     // per generation g: DIM_GEN0 + DIMS_PER_GEN * g + offset
    DIMS_PER_GEN = 8,
    OFF_STRATEGY = 0,
    OFF_BSDF = 1,     // 2 ids
    OFF_COMPONENT = 3,
    OFF_LIGHT_CHOICE = 4,
    OFF_LIGHT = 5,    // 2 ids
    OFF_RR = 7
};

// sampler modes (liar_render_desc.sampler, include/liar_gpu.h)
//   default        Stratifier (samplers/stratifier.cpp:163-180): screen and lens samples on the
//                  sqrt(spp) x sqrt(spp) grid of 2D strata when spp is a square
//   LATIN          LatinHypercube (samplers/latin_hypercube.cpp): screen and lens axes stratified
//                  separately over the spp samples, like every other dimension
//   NOT_JITTERED   `jittered = False`: every stratified value sits at its stratum's centre (the
//                  reference's jitter() returns 0.5, stratifier.h:90)
enum : uint32_t { SAMPLER_LATIN = 1u, SAMPLER_NOT_JITTERED = 2u };

struct SampleKey {
    uint64_t seed;
    uint32_t pixel, sample, spp;
    uint32_t mode = 0;
};

LS_HD uint64_t dim_hash(const SampleKey& k, uint32_t dim) {
    return mix64(k.seed ^ mix64(((uint64_t)k.pixel << 32) | (uint64_t)dim));
}
LS_HD float dim_jitter(const SampleKey& k, uint64_t hd) {
    return to_unit(mix64(hd + 0xd1b54a32d192ed03ull * ((uint64_t)k.sample + 1)));
}

LS_HD float sample_dim(const SampleKey& k, uint32_t dim, bool stratified) {
    const uint64_t hd = dim_hash(k, dim);
    if (!stratified) return dim_jitter(k, hd);
    const float jitter = (k.mode & SAMPLER_NOT_JITTERED) ? 0.5f : dim_jitter(k, hd);
    if (k.spp <= 1) return jitter;
    const uint32_t s = permute_index(k.sample, k.spp, hd);
    const float u = ((float)s + jitter) / (float)k.spp;
    return u < 1.0f ? u : 0.99999994f;
}

// exact integer square root of small counts
LS_HD uint32_t isqrt_u32(uint32_t n) {
    uint32_t r = 0;
    while ((r + 1) * (r + 1) <= n) ++r;
    return r;
}

// the 2D sample of dimensions (dim, dim + 1): one of the spp = n^2 cells of the n x n grid per
// sample (a bijection keyed by the pixel and dim), jittered within the cell; LatinHypercube
// mode, or a count that is not a square, stratifies the two axes separately
LS_HD void sample_2d(const SampleKey& k, uint32_t dim, float& x, float& y) {
    const uint32_t n = k.spp > 1 ? isqrt_u32(k.spp) : 1u;
    if ((k.mode & SAMPLER_LATIN) || k.spp <= 1 || n * n != k.spp) {
        x = sample_dim(k, dim, true);
        y = sample_dim(k, dim + 1, true);
        return;
    }
    const uint64_t hx = dim_hash(k, dim), hy = dim_hash(k, dim + 1);
    const uint32_t s = permute_index(k.sample, k.spp, hx);
    const bool jit = !(k.mode & SAMPLER_NOT_JITTERED);
    const float jx = jit ? dim_jitter(k, hx) : 0.5f, jy = jit ? dim_jitter(k, hy) : 0.5f;
    const float u = ((float)(s % n) + jx) / (float)n, v = ((float)(s / n) + jy) / (float)n;
    x = u < 1.0f ? u : 0.99999994f;
    y = v < 1.0f ? v : 0.99999994f;
}

}  // namespace liar_gpu
