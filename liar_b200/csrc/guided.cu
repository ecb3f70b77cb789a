// guided.cu -- the AdjointPhotonTracer estimator with a learned guide as a third sampling
// technique, trained online on its own samples (no reference counterpart; the estimator without
// the guide is src/liar/tracers/adjoint_photon_tracer.cpp:84-292, as in render.cu).
//
// Per wave of paths: raygen -> per bounce [trace, (guide inputs of the diffuse and glossy
// vertices, guide network over the queue on the tensor cores), shade]; the shade kernel is one
// thread per queue entry and reads its vertex's mixture when it makes the scattering decision:
//   directional strategy (probability s = 0.5 at diffuse/glossy vertices): guide with probability
//   c, else BSDF; density p_d = c q + (1 - c) p_bsdf
//   light strategy (probability 1 - s): as the reference
// weighted by the power heuristic between s p_d and (1 - s) p_light (one-sample MIS). With c = 0
// every float operation is the one of render.cu, so the images agree to rounding.
// Training records (vertex, direction, integrand / density) are written per scattering event and
// completed when the wave ends: weight = (L_end - L_at_vertex) * p_chosen / (w_mis T_vertex p_mix),
// the sampled integrand f cos L_in over the density p_mix of the whole one-sample mixture. Paths
// are numbered sample-major, so a training wave of whole passes covers the whole image; when the
// record buffer cannot hold every candidate, a random subset is kept; the records with a positive
// weight are stride-permuted before the Adam steps so that each batch mixes all generations.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "../../include/liar_gpu.h"
#include "ctx.h"
#include "guide_mlp.cuh"
#include "render_dev.cuh"

using namespace liar_gpu;
using namespace liar_gpu::rt;
using namespace liar_gpu::guide;

namespace liar_gpu {
namespace rt {
const DScene& scene_dscene(const liar_gpu_scene* s);
const liar_gpu_mesh* scene_mesh(const liar_gpu_scene* s);
int scene_device(const liar_gpu_scene* s);
}  // namespace rt
namespace guide {
const liar_guide_config& guide_config(const liar_gpu_guide* g);
int guide_device(const liar_gpu_guide* g);
int guide_train(liar_gpu_ctx* ctx, liar_gpu_guide* g, const float* d_records, const uint32_t* d_count, size_t n_max,
                int apply, float* d_grad_out, float* d_loss_out, cudaStream_t st);
void guide_count(liar_gpu_guide* g, unsigned long long records, unsigned long long guided, unsigned long long passes);
unsigned long long guide_steps(const liar_gpu_guide* g);
int guide_eval(liar_gpu_ctx* ctx, const liar_gpu_guide* G, const float* d_inputs, size_t n, float* d_mixture,
               int stride, cudaStream_t st);
}  // namespace guide
}  // namespace liar_gpu

namespace {

constexpr int kRawRecord = 15;  // position 3, normal 3, direction to the previous vertex 3, sampled direction 3,
                                // path slot, radiance before, scale
constexpr int kTrainRecord = 13;
constexpr uint32_t kDimGuide = 0x100000u;  // per generation g: kDimGuide + 4 g + {choice, lobe, cosine, azimuth}

struct GPaths {
    float* lam;
    float* lam_pdf;
    float* T;
    float* L;
    float* alpha;
    int32_t* gen;
};

struct GQueue {
    liar_ray* rays;
    uint32_t* path;
    uint32_t* count;
};

struct GParams {
    liar_camera cam;
    int width, height, spp, max_gen, max_depth;
    uint32_t sampler;       // SAMPLER_* mode bits (sampler.h)
    uint64_t seed;
    uint64_t first_path;    // global index (sample * pixels + pixel) of the wave's first path
    uint32_t npix;
    float guide_prob;       // c (0: guide off)
    float light_prob;       // light-sampling share at guided vertices
    int train;
    float rec_keep;         // probability that a candidate training record is kept
    float box_lo[3], box_inv[3];
    float* records;         // raw records
    uint32_t* rec_count;    // [0] kept records [2] candidates
    uint32_t rec_cap;
    unsigned long long* stats;  // [0] paths [1] segments [2] hits [3] guided vertices
    FilmSpec film;
};

// Paths are numbered sample-major: a run of npix consecutive paths is one sample of every pixel,
// so a training wave of whole passes sees the whole image.
__device__ __forceinline__ SampleKey gkey(const GParams& W, uint32_t slot) {
    const uint64_t g = W.first_path + slot;
    SampleKey k;
    k.seed = W.seed;
    k.pixel = (uint32_t)(g % (uint64_t)W.npix);
    k.sample = (uint32_t)(g / (uint64_t)W.npix);
    k.spp = (uint32_t)W.spp;
    k.mode = W.sampler;
    return k;
}

// a uniform number in [0, 1) per (path, generation) that decides whether a candidate training
// record is kept: the kept records are an unbiased thinning of all of the wave's vertices
__device__ __forceinline__ float record_lottery(const GParams& W, uint32_t slot, int gen) {
    const uint64_t h = mix64(W.seed ^ mix64(((W.first_path + slot) << 8) | (uint64_t)(gen & 0xff)) ^ 0x7f4a7c159e3779b9ull);
    return (float)(h >> 40) * (1.0f / 16777216.0f);
}

__device__ __forceinline__ void gqueue_push(const GQueue& q, bool want, const liar_ray& r, uint32_t path) {
    const uint32_t mask = __ballot_sync(0xffffffffu, want);
    if (mask == 0) return;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(q.count, (uint32_t)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (want) {
        const uint32_t slot = base + __popc(mask & ((1u << lane) - 1u));
        float4* dst = reinterpret_cast<float4*>(q.rays + slot);
        dst[0] = make_float4(r.ox, r.oy, r.oz, r.tmin);
        dst[1] = make_float4(r.dx, r.dy, r.dz, r.tmax);
        q.path[slot] = path;
    }
}

__device__ void gsplat(const DScene& S, const GParams& W, uint32_t slot, float lam, float lam_pdf, float L, float alpha) {
    float3 xyz = mk(0, 0, 0);
    if (lam_pdf > 0.0f) {
        const float s = L / lam_pdf;
        const float3 c = observer_sensitivity(S, lam);
        xyz = mk(s * c.x, s * c.y, s * c.z);
    }
    film_splat(W.film, gkey(W, slot), xyz, alpha);
}

__global__ void __launch_bounds__(256) k_g_raygen(DScene S, GParams W, GPaths P, GQueue out, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool want = false;
    liar_ray r{};
    if (i < n) {
        const SampleKey k = gkey(W, i);
        float lpdf;
        const float lam = observer_sample(S, sample_dim(k, DIM_LAMBDA, true), lpdf);
        r = camera_ray(W.cam, k, W.width, W.height);
        P.lam[i] = lam;
        P.lam_pdf[i] = lpdf;
        P.T[i] = 1.0f;
        P.L[i] = 0.0f;
        P.alpha[i] = 0.0f;
        P.gen[i] = 0;
        want = true;
    }
    gqueue_push(out, want, r, i);
}

constexpr int kShadeThreads = 128;

// the guide's inputs for every queue entry that sits on a diffuse or glossy surface (position,
// shading normal, direction to the previous vertex; zeros elsewhere)
__global__ void __launch_bounds__(128) k_g_prep(DScene S, GQueue in, const liar_hit* __restrict__ hits, uint32_t n_in,
                                                float* __restrict__ gin) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n_in) return;
    float x[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const liar_hit h = hits[q];
    if (h.prim >= 0) {
        const float4 r0 = reinterpret_cast<const float4*>(in.rays + q)[0];
        const float4 r1 = reinterpret_cast<const float4*>(in.rays + q)[1];
        const int obj = prim_object(S, (uint32_t)h.prim);
        const int mi = S.obj_mat[obj];
        if (mi >= 0) {
            const int type = S.mats[mi].type;
            if (type == LIAR_MAT_LAMBERT || type == LIAR_MAT_COOK_TORRANCE || type == LIAR_MAT_WALTER) {
                const HitContext HC = hit_context(S, mk(r0.x, r0.y, r0.z), mk(r1.x, r1.y, r1.z), (uint32_t)h.prim, h.t);
                x[0] = HC.target.x;
                x[1] = HC.target.y;
                x[2] = HC.target.z;
                x[3] = HC.N.x;
                x[4] = HC.N.y;
                x[5] = HC.N.z;
                x[6] = -r1.x;
                x[7] = -r1.y;
                x[8] = -r1.z;
            }
        }
    }
    float* dst = gin + (size_t)q * 9;
#pragma unroll
    for (int c = 0; c < 9; ++c) dst[c] = x[c];
}

template <bool TEX>
__global__ void __launch_bounds__(kShadeThreads) k_g_shade(DScene S, GParams W, GPaths P, GQueue in,
                                                           const liar_hit* __restrict__ hits, uint32_t n_in, GQueue out,
                                                           const float* __restrict__ gmix) {
    const int lane = threadIdx.x & 31;
    const bool guide_on = W.guide_prob > 0.0f;
    unsigned long long segs = 0, n_hit = 0, n_guided = 0;
    {
        const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
        const bool valid = q < n_in;
        uint32_t p = 0;
        float4 r0 = make_float4(0, 0, 0, 0), r1 = make_float4(0, 0, 1, 0);
        liar_hit h{-1, 0.0f};
        HitContext HC;
        HC.mat = -1;
        HC.light = -1;
        bool surface = false, guidable = false;
        liar_material M{};
        if (valid) {
            p = in.path[q];
            r0 = reinterpret_cast<const float4*>(in.rays + q)[0];
            r1 = reinterpret_cast<const float4*>(in.rays + q)[1];
            h = hits[q];
            if (h.prim >= 0) {
                HC = hit_context(S, mk(r0.x, r0.y, r0.z), mk(r1.x, r1.y, r1.z), (uint32_t)h.prim, h.t);
                surface = HC.mat >= 0 && S.mats[HC.mat].type != LIAR_MAT_NONE;
                if (surface) {
                    M = S.mats[HC.mat];
                    guidable = M.type == LIAR_MAT_LAMBERT || M.type == LIAR_MAT_COOK_TORRANCE ||
                               M.type == LIAR_MAT_WALTER;
                }
            }
        }
        // the guide's mixture at this vertex (computed by the network for the whole queue), read
        // where it is used (only when the vertex is guided) rather than held in registers
        const float* __restrict__ mix = gmix + (size_t)q * kMixRender;
        // ---- shading (render.cu's k_shade with the guide as a third technique)
        bool want = false;
        liar_ray nr{};
        bool rec_want = false, rec_cand = false;
        float rec[kRawRecord];
        if (valid) {
            ++segs;
            const float3 o = mk(r0.x, r0.y, r0.z), d = mk(r1.x, r1.y, r1.z);
            const SampleKey key = gkey(W, p);
            const int gen = P.gen[p];
            // the camera vertex carries the camera's ray differentials (texture filtering)
            if (TEX && surface && gen == 0) camera_footprint(S, HC, (uint32_t)h.prim, W.cam, key, W.width, W.height);
            float T = P.T[p], L = P.L[p];
            const float lam = P.lam[p];
            bool alive = false;
            float3 next_o = mk(0, 0, 0), next_d = mk(0, 0, 1);
            float next_tmin = kTol, next_tmax = INFINITY;
            if (h.prim < 0) {
                if (S.sky_light >= 0 && S.sky_distance > r0.w * (1.0f + kTol) && S.sky_distance < r1.w * (1.0f - kTol)) {
                    if (gen == 0) P.alpha[p] = 1.0f;
                    if (gen > 0) L += T * spec_eval(S, S.lights[S.sky_light].spectrum, lam, false);
                }
            } else {
                ++n_hit;
                if (gen == 0) P.alpha[p] = 1.0f;
                const int light = HC.light, mi = HC.mat;
                const float3 target = HC.target, ng = HC.ng, N = HC.N, u = HC.u, v = HC.v;
                if (gen > 0 && light >= 0) L += T * spec_eval(S, S.lights[light].spectrum, lam, false);
                const bool shader_emits = gen == 0 || light < 0;  // as render.cu
                if (mi < 0) {
                    alive = true;  // no shader: continue through
                    next_o = o;
                    next_d = d;
                    next_tmin = h.t + kTol;
                    next_tmax = r1.w;
                } else if (!surface) {
                    // a shader without a BSDF: its emission, and the path ends
                    if (shader_emits && S.mats[mi].emission >= 0) L += T * spec_eval(S, S.mats[mi].emission, lam, false);
                } else {
                    if (shader_emits && M.emission >= 0) L += T * spec_eval(S, M.emission, lam, false);
                    const Bsdf B = make_bsdf<TEX>(S, M, HC, lam);
                    const float3 md = -d;
                    float3 wi = mk(dot(md, u), dot(md, v), dot(md, N));
                    wi.z = fmaxf(wi.z, kEps);
                    const bool strat = gen < W.max_gen;
                    const uint32_t base = DIM_GEN0 + DIMS_PER_GEN * (uint32_t)gen;
                    const bool smooth = has_caps(B.caps, CAP_DIFF) || has_caps(B.caps, CAP_GLOSSY);
                    const bool guided = guide_on && guidable && smooth;
                    const float strategy_pdf = smooth ? (guided ? 1.0f - W.light_prob : 0.5f) : 1.0f;
                    const float c = guided ? W.guide_prob : 0.0f;
                    const uint32_t gbase = kDimGuide + 4u * (uint32_t)gen;
                    float3 wo = mk(0, 0, 1);
                    float3 wd = mk(0, 0, 1);
                    float value = 0.0f, pdf_s = 0.0f, w_mis = 0.0f, p_mix = 0.0f;
                    bool ok = false;
                    if (sample_dim(key, base + OFF_STRATEGY, strat) < strategy_pdf) {
                        float p_dir = 0.0f;
                        if (c > 0.0f && sample_dim(key, gbase, false) < c) {
                            // the guide
                            ++n_guided;
                            float gx, gy, gz;
                            mixture_sample(mix, sample_dim(key, gbase + 1, false), sample_dim(key, gbase + 2, false),
                                           sample_dim(key, gbase + 3, false), gx, gy, gz);
                            wd = mk(gx, gy, gz);
                            wo = mk(dot(wd, u), dot(wd, v), dot(wd, N));
                            const BsdfOut be = bsdf_evaluate(B, wi, wo, CAP_ALL);
                            p_dir = c * mixture_pdf_render(mix, gx, gy, gz) + (1.0f - c) * be.pdf;
                            value = be.value;
                            ok = p_dir > 0.0f && value != 0.0f;
                        } else {
                            const BsdfSample bs = bsdf_sample(B, wi, sample_dim(key, base + OFF_BSDF, strat),
                                                              sample_dim(key, base + OFF_BSDF + 1, strat),
                                                              sample_dim(key, base + OFF_COMPONENT, strat), CAP_ALL);
                            if (bs.ok()) {
                                wo = bs.wo;
                                wd = bs.wo.x * u + bs.wo.y * v + bs.wo.z * N;
                                const float qd = c > 0.0f ? mixture_pdf_render(mix, wd.x, wd.y, wd.z) : 0.0f;
                                p_dir = c > 0.0f ? c * qd + (1.0f - c) * bs.pdf : bs.pdf;
                                value = bs.value;
                                ok = true;
                            }
                        }
                        if (ok) {
                            pdf_s = p_dir * strategy_pdf;
                            float pl = 0.0f;
                            for (int l = 0; l < S.n_lights; ++l) {
                                const LightEmission e = light_emission(S, l, target, wd, lam);
                                if (e.pdf > 0.0f) pl += light_choice_pdf(S, l) * e.pdf;
                            }
                            pl *= (1.0f - strategy_pdf);
                            w_mis = power_heuristic(pdf_s, pl);
                            value *= w_mis;
                            ok = pdf_s > 0.0f && value != 0.0f;
                            p_mix = pdf_s + pl;
                        }
                    } else if (S.n_lights > 0) {
                        const float uc = sample_dim(key, base + OFF_LIGHT_CHOICE, strat);
                        int k = lower_bound_f(S.light_cdf, S.n_lights, uc);
                        if (k > S.n_lights - 1) k = S.n_lights - 1;
                        const float pc = light_choice_pdf(S, k);
                        if (pc > 0.0f) {
                            const LightSample ls = light_sample(S, k, target, sample_dim(key, base + OFF_LIGHT, strat),
                                                                sample_dim(key, base + OFF_LIGHT + 1, strat), lam);
                            if (ls.pdf > 0.0f) {
                                float pdf = pc * ls.pdf;
                                for (int l = 0; l < S.n_lights; ++l) {
                                    if (l == k) continue;
                                    const LightEmission e = light_emission(S, l, target, ls.dir, lam);
                                    if (e.pdf > 0.0f) pdf += light_choice_pdf(S, l) * e.pdf;
                                }
                                pdf *= (1.0f - strategy_pdf);
                                const float3 lwo = mk(dot(ls.dir, u), dot(ls.dir, v), dot(ls.dir, N));
                                const BsdfOut be = bsdf_evaluate(B, wi, lwo, CAP_ALL);
                                if (be.pdf > 0.0f && be.value != 0.0f) {
                                    const float p_dir =
                                        c > 0.0f ? c * mixture_pdf_render(mix, ls.dir.x, ls.dir.y, ls.dir.z) + (1.0f - c) * be.pdf
                                                 : be.pdf;
                                    wo = lwo;
                                    wd = ls.dir;
                                    w_mis = power_heuristic(pdf, p_dir * strategy_pdf);
                                    value = be.value * w_mis;
                                    pdf_s = pdf;
                                    ok = pdf_s > 0.0f && value != 0.0f;
                                    p_mix = pdf + p_dir * strategy_pdf;
                                }
                            }
                        }
                    }
                    if (ok) {
                        const float cos_t = wo.z;
                        next_o = target + ((cos_t > 0.0f ? 10.0f : -10.0f) * kTol) * ng;
                        next_d = wo.x * u + wo.y * v + wo.z * N;
                        next_tmin = kTol;
                        next_tmax = INFINITY;
                        if (W.train && guidable && strategy_pdf < 1.0f && T > 0.0f && w_mis > 0.0f && p_mix > 0.0f) {
                            rec_cand = true;
                            rec_want = record_lottery(W, p, gen) < W.rec_keep;
                            rec[0] = target.x;
                            rec[1] = target.y;
                            rec[2] = target.z;
                            rec[3] = N.x;
                            rec[4] = N.y;
                            rec[5] = N.z;
                            rec[6] = -d.x;
                            rec[7] = -d.y;
                            rec[8] = -d.z;
                            rec[9] = wd.x;
                            rec[10] = wd.y;
                            rec[11] = wd.z;
                            rec[12] = __uint_as_float(p);
                            rec[13] = L;
                            rec[14] = pdf_s / (w_mis * T * p_mix);
                        }
                        T *= value * (fabsf(cos_t) / pdf_s);
                        alive = true;
                    }
                }
            }
            if (alive) {
                const int ng1 = gen + 1;
                if (W.max_depth > 0 && ng1 >= W.max_depth) {
                    alive = false;
                } else if (ng1 >= W.max_gen) {
                    const float ur = sample_dim(key, DIM_GEN0 + DIMS_PER_GEN * (uint32_t)ng1 + OFF_RR, false);
                    if (ur < 0.5f) T /= 0.5f;
                    else alive = false;
                }
            }
            if (alive) {
                P.T[p] = T;
                P.L[p] = L;
                P.gen[p] = gen + 1;
                nr = liar_ray{next_o.x, next_o.y, next_o.z, next_tmin, next_d.x, next_d.y, next_d.z, next_tmax};
                want = true;
            } else {
                P.L[p] = L;  // the radiance at the end of the path completes its training records
                gsplat(S, W, p, lam, P.lam_pdf[p], L, P.alpha[p]);
            }
        }
        gqueue_push(out, want, nr, p);
        // training records, one atomic per warp
        const uint32_t cmask = __ballot_sync(0xffffffffu, rec_cand);
        if (cmask && (uint32_t)lane == __ffs(cmask) - 1) atomicAdd(W.rec_count + 2, (uint32_t)__popc(cmask));
        const uint32_t rmask = __ballot_sync(0xffffffffu, rec_want);
        if (rmask) {
            const uint32_t leader = __ffs(rmask) - 1;
            uint32_t rb = 0;
            if ((uint32_t)lane == leader) rb = atomicAdd(W.rec_count, (uint32_t)__popc(rmask));
            rb = __shfl_sync(0xffffffffu, rb, leader);
            if (rec_want) {
                const uint32_t slot = rb + __popc(rmask & ((1u << lane) - 1u));
                if (slot < W.rec_cap) {
                    float* dst = W.records + (size_t)slot * kRawRecord;
                    for (int c = 0; c < kRawRecord; ++c) dst[c] = rec[c];
                }
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        segs += __shfl_down_sync(0xffffffffu, segs, o);
        n_hit += __shfl_down_sync(0xffffffffu, n_hit, o);
        n_guided += __shfl_down_sync(0xffffffffu, n_guided, o);
    }
    if (lane == 0 && segs) {
        atomicAdd(W.stats + 1, segs);
        atomicAdd(W.stats + 2, n_hit);
        if (n_guided) atomicAdd(W.stats + 3, n_guided);
    }
}

// completes the wave's records: weight = (L_end - L_vertex) * scale; keeps the positive ones
__global__ void k_g_finalize(const float* __restrict__ raw, const uint32_t* __restrict__ raw_count, uint32_t raw_cap,
                             const float* __restrict__ L_end, float* __restrict__ train, uint32_t* train_count,
                             uint32_t train_cap) {
    const uint32_t n = min(*raw_count, raw_cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float* r = raw + (size_t)i * kRawRecord;
        const uint32_t p = __float_as_uint(r[12]);
        const float w = (L_end[p] - r[13]) * r[14];
        if (w > 0.0f && isfinite(w)) {
            const uint32_t slot = atomicAdd(train_count, 1u);
            if (slot < train_cap) {
                float* d = train + (size_t)slot * kTrainRecord;
                for (int c = 0; c < 12; ++c) d[c] = r[c];
                d[12] = w;
            }
        }
    }
}

// out[(i * A) mod m] = in[i]: a stride permutation of the training records (A prime and > m, so it
// is a bijection), which spreads every batch over all generations of the wave; the raw records are
// in order of generation
__global__ void k_g_shuffle(const float* __restrict__ in, float* __restrict__ out, uint32_t m, uint32_t A) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const uint32_t j = (uint32_t)(((uint64_t)i * A) % m);
        const float* s = in + (size_t)i * kTrainRecord;
        float* d = out + (size_t)j * kTrainRecord;
        for (int c = 0; c < kTrainRecord; ++c) d[c] = s[c];
    }
}

struct GuidedBuffers {
    size_t cap = 0;       // paths per wave
    size_t rec_cap = 0;   // raw records per wave
    void* mem = nullptr;
    GPaths P{};
    GQueue q[2]{};
    liar_hit* hits = nullptr;
    float* raw = nullptr;
    float* train = nullptr;
    float* shuffled = nullptr;  // the training records in stride-permuted order
    float* gin = nullptr;   // guide inputs per queue entry (9 floats)
    float* gmix = nullptr;  // guide mixtures per queue entry (40 floats)
    uint32_t* counters = nullptr;            // [0] raw records [1] training records [2] candidates
    unsigned long long* stats = nullptr;     // [0..3]
    uint32_t* h_count = nullptr;             // pinned, 4 words
};

GuidedBuffers* guided_buffers(liar_gpu_ctx* ctx) {
    for (auto& ext : ctx->extensions)
        if (ext.first == "guided") return static_cast<GuidedBuffers*>(ext.second);
    GuidedBuffers* gb = new GuidedBuffers();
    ctx->extensions.emplace_back("guided", gb);
    ctx->on_destroy.push_back([gb]() {
        if (gb->mem) cudaFree(gb->mem);
        if (gb->h_count) cudaFreeHost(gb->h_count);
        delete gb;
    });
    return gb;
}

int ensure_guided_buffers(liar_gpu_ctx* ctx, GuidedBuffers* gb, size_t n, size_t rec_cap) {
    if (!gb->h_count) {
        cudaError_t e = cudaMallocHost((void**)&gb->h_count, 4 * sizeof(uint32_t));
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "guided render host buffers");
    }
    if (gb->cap >= n && gb->rec_cap >= rec_cap) return LIAR_OK;
    // grow, keeping what earlier calls needed (training and rendering calls alternate)
    n = std::max(n, gb->cap);
    rec_cap = std::max(rec_cap, gb->rec_cap);
    if (gb->mem) cudaFree(gb->mem);
    gb->mem = nullptr;
    gb->cap = gb->rec_cap = 0;
    const size_t bytes =
        n * (6 * 4 + 2 * (32 + 4) + 8 + (9 + kMixRender) * 4) + rec_cap * (kRawRecord + 2 * kTrainRecord) * 4 + 8192;
    cudaError_t e = cudaMalloc(&gb->mem, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return ctx_cuda(ctx, e, "guided render buffers");
    }
    char* p = static_cast<char*>(gb->mem);
    auto take = [&](size_t b) {
        char* r = p;
        p += (b + 255) & ~size_t(255);
        return r;
    };
    gb->q[0].rays = reinterpret_cast<liar_ray*>(take(n * 32));
    gb->q[1].rays = reinterpret_cast<liar_ray*>(take(n * 32));
    gb->hits = reinterpret_cast<liar_hit*>(take(n * 8));
    gb->q[0].path = reinterpret_cast<uint32_t*>(take(n * 4));
    gb->q[1].path = reinterpret_cast<uint32_t*>(take(n * 4));
    gb->P.lam = reinterpret_cast<float*>(take(n * 4));
    gb->P.lam_pdf = reinterpret_cast<float*>(take(n * 4));
    gb->P.T = reinterpret_cast<float*>(take(n * 4));
    gb->P.L = reinterpret_cast<float*>(take(n * 4));
    gb->P.alpha = reinterpret_cast<float*>(take(n * 4));
    gb->P.gen = reinterpret_cast<int32_t*>(take(n * 4));
    gb->gin = reinterpret_cast<float*>(take(n * 9 * 4));
    gb->gmix = reinterpret_cast<float*>(take(n * kMixRender * 4));
    gb->raw = reinterpret_cast<float*>(take(rec_cap * kRawRecord * 4));
    gb->train = reinterpret_cast<float*>(take(rec_cap * kTrainRecord * 4));
    gb->shuffled = reinterpret_cast<float*>(take(rec_cap * kTrainRecord * 4));
    gb->q[0].count = reinterpret_cast<uint32_t*>(take(4));
    gb->q[1].count = reinterpret_cast<uint32_t*>(take(4));
    gb->counters = reinterpret_cast<uint32_t*>(take(16));
    gb->stats = reinterpret_cast<unsigned long long*>(take(4 * 8));
    gb->cap = n;
    gb->rec_cap = rec_cap;
    return LIAR_OK;
}

}  // namespace

extern "C" int liar_gpu_render_guided_device(liar_gpu_ctx* ctx, const liar_gpu_scene* scene, liar_gpu_guide* guide,
                                             const liar_render_desc* desc, int train, float* d_film, void* stream) {
    if (!ctx) return LIAR_ERR_INVALID;
    if (!scene || !guide || !desc || !d_film) return ctx_fail(ctx, LIAR_ERR_INVALID, "null scene, guide, description or film");
    if (scene_device(scene) != ctx->device || guide_device(guide) != ctx->device)
        return ctx_fail(ctx, LIAR_ERR_INVALID, "scene or guide lives on another device");
    const liar_render_desc& R = *desc;
    if (R.width <= 0 || R.height <= 0 || R.spp <= 0) return ctx_fail(ctx, LIAR_ERR_INVALID, "empty image or no samples");
    if (R.max_ray_generation < 0) return ctx_fail(ctx, LIAR_ERR_INVALID, "max_ray_generation must be >= 0");
    if (R.tracer != LIAR_TRACER_ADJOINT_PHOTON) return ctx_fail(ctx, LIAR_ERR_UNSUPPORTED, "tracer %d", R.tracer);
    if (const char* m = film_desc_error(R)) return ctx_fail(ctx, LIAR_ERR_INVALID, "%s", m);
    const uint64_t npix = (uint64_t)R.width * R.height;
    if (npix >= (1ull << 32)) return ctx_fail(ctx, LIAR_ERR_INVALID, "image too large");
    const uint64_t total = npix * (uint64_t)R.spp;
    // paths per wave: without training as many as fit (4M); when training, the guide learns after
    // every wave, so a wave is a whole number of passes over the image, about 2M paths
    GuidedBuffers* gb = guided_buffers(ctx);
    uint64_t wave;
    if (R.wave_paths > 0) wave = (uint64_t)R.wave_paths;
    else if (train) wave = npix * std::max<uint64_t>(1, (1ull << 21) / npix);
    else wave = gb->cap >= (1u << 20) ? gb->cap : (1ull << 22);  // reuse the buffers of earlier waves
    wave = std::min<uint64_t>(std::min<uint64_t>(wave, total), 1ull << 26);
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    const liar_guide_config& cfg = guide_config(guide);
    const uint32_t batch = cfg.batch_records > 0 ? (uint32_t)cfg.batch_records : 65536u;
    const int steps = cfg.steps_per_pass > 0 ? cfg.steps_per_pass : 4;
    // raw records: room for about 2.5 candidates per path (at most 2^25 records); only the records
    // whose path found light after the vertex train the guide, usually a few percent, so every
    // candidate is kept while the buffer has room, and when it has not, a random subset (the keep
    // probability follows the previous wave's candidates per path, with 20% slack)
    const size_t rec_cap = train ? std::min<size_t>(std::max<size_t>((size_t)wave * 5 / 2, (size_t)batch * steps), 1ull << 25) : 0;
    const size_t rec_target = rec_cap - rec_cap / 5;
    rc = ensure_guided_buffers(ctx, gb, (size_t)wave, rec_cap);
    if (rc) return rc;
    cudaError_t e = cudaMemsetAsync(gb->stats, 0, 4 * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "reset statistics");
    GParams W;
    W.cam = R.camera;
    W.width = R.width;
    W.height = R.height;
    W.spp = R.spp;
    W.max_gen = R.max_ray_generation;
    W.max_depth = R.max_depth;
    W.sampler = (uint32_t)R.sampler;
    W.seed = mix64(R.seed ^ mix64(0x51ed270b27ad0e0dull + (uint64_t)(uint32_t)R.first_sample));
    W.npix = (uint32_t)npix;
    W.film = film_spec(d_film, R);
    W.train = train ? 1 : 0;
    for (int k = 0; k < 3; ++k) {
        W.box_lo[k] = cfg.bounds_lo[k];
        W.box_inv[k] = 1.0f / (cfg.bounds_hi[k] - cfg.bounds_lo[k]);
    }
    W.records = gb->raw;
    W.rec_count = gb->counters;
    W.rec_cap = (uint32_t)rec_cap;
    W.stats = gb->stats;
    const DScene& S = scene_dscene(scene);
    const liar_gpu_mesh* mesh = scene_mesh(scene);
    unsigned long long records_total = 0;
    double candidates_per_path = 2.0;
    for (uint64_t first = 0; first < total; first += wave) {
        if (ctx_cancel_requested(ctx)) return ctx_cancelled(ctx, st);
        const uint32_t n = (uint32_t)std::min<uint64_t>(wave, total - first);
        W.first_path = first;
        W.rec_keep = (float)std::min(1.0, (double)rec_target / ((double)n * candidates_per_path));
        // an untrained guide is not sampled: the first training wave renders with BSDF and lights only
        W.guide_prob = (train && guide_steps(guide) == 0) ? 0.0f : cfg.guide_probability;
        W.light_prob = cfg.light_probability > 0.0f ? cfg.light_probability : 0.5f;
        const bool guide_on = W.guide_prob > 0.0f;
        e = cudaMemsetAsync(gb->q[0].count, 0, 4, st);
        if (e == cudaSuccess && train) e = cudaMemsetAsync(gb->counters, 0, 12, st);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "reset queue");
        k_g_raygen<<<(n + 255) / 256, 256, 0, st>>>(S, W, gb->P, gb->q[0], n);
        uint32_t n_in = n;
        int cur = 0;
        for (int bounce = 0; n_in > 0; ++bounce) {
            if (bounce > 4096) return ctx_fail(ctx, LIAR_ERR_TIMEOUT, "paths did not terminate after 4096 bounces");
            if (ctx_cancel_requested(ctx)) return ctx_cancelled(ctx, st);
            rc = trace_mesh_internal(ctx, mesh, gb->q[cur].rays, n_in, gb->hits, 0, st, kCounterWord + 8);
            if (rc) return rc;
            e = cudaMemsetAsync(gb->q[cur ^ 1].count, 0, 4, st);
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "reset queue");
            if (guide_on) {
                // the guide network over the queue's diffuse and glossy vertices
                k_g_prep<<<(n_in + 127) / 128, 128, 0, st>>>(S, gb->q[cur], gb->hits, n_in, gb->gin);
                rc = guide_eval(ctx, guide, gb->gin, n_in, gb->gmix, kMixRender, st);
                if (rc) return rc;
            }
            (S.n_tex > 0 ? k_g_shade<true> : k_g_shade<false>)<<<(n_in + kShadeThreads - 1) / kShadeThreads, kShadeThreads, 0, st>>>(
                S, W, gb->P, gb->q[cur], gb->hits, n_in, gb->q[cur ^ 1], gb->gmix);
            e = cudaGetLastError();
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "guided shade launch");
            cur ^= 1;
            e = cudaMemcpyAsync(gb->h_count, gb->q[cur].count, 4, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "queue size");
            n_in = gb->h_count[0];
        }
        if (train) {
            k_g_finalize<<<ctx->num_sms * 4, 256, 0, st>>>(gb->raw, gb->counters, (uint32_t)rec_cap, gb->P.L, gb->train,
                                                           gb->counters + 1, (uint32_t)rec_cap);
            e = cudaMemcpyAsync(gb->h_count, gb->counters, 12, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "training records");
            const uint32_t n_train = std::min<uint32_t>(gb->h_count[1], (uint32_t)rec_cap);
            if (gb->h_count[2] > 0) candidates_per_path = (double)gb->h_count[2] / (double)n;
            records_total += n_train;
            if (n_train > 0) {
                k_g_shuffle<<<ctx->num_sms * 4, 256, 0, st>>>(gb->train, gb->shuffled, n_train, 2147483647u);
                e = cudaGetLastError();
                if (e != cudaSuccess) return ctx_cuda(ctx, e, "shuffle launch");
                for (int s = 0; s < steps; ++s) {
                    const uint32_t first = (uint32_t)(((uint64_t)s * batch) % n_train);
                    const uint32_t cnt = std::min<uint32_t>(batch, n_train - first);
                    rc = guide_train(ctx, guide, gb->shuffled + (size_t)first * kTrainRecord, nullptr, cnt, 1, nullptr,
                                     nullptr, st);
                    if (rc) return rc;
                }
            }
        }
    }
    unsigned long long stats[4];
    e = cudaMemcpyAsync(stats, gb->stats, sizeof(stats), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "guided render statistics");
    guide_count(guide, records_total, stats[3], (unsigned long long)R.spp);
    stats[0] = npix * (uint64_t)R.spp;
    e = cudaMemcpyAsync(gb->stats, stats, 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "guided render statistics");
    return ctx_check_status(ctx);
}

extern "C" int liar_gpu_render_guided_stats(const liar_gpu_ctx* ctx, unsigned long long* out4) {
    if (!ctx || !out4) return LIAR_ERR_INVALID;
    for (auto& ext : ctx->extensions)
        if (ext.first == "guided") {
            GuidedBuffers* gb = static_cast<GuidedBuffers*>(ext.second);
            if (!gb->stats) break;
            if (cudaMemcpy(out4, gb->stats, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost) != cudaSuccess) {
                cudaGetLastError();
                return LIAR_ERR_CUDA;
            }
            return LIAR_OK;
        }
    for (int k = 0; k < 4; ++k) out4[k] = 0;
    return LIAR_OK;
}
