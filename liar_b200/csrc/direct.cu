// direct.cu -- the DirectLighting tracer on sm_100a (src/liar/tracers/direct_lighting.cpp), with
// RayTracer::estimateLightContribution (src/liar/kernel/ray_tracer.cpp:188-276) as its direct term.
//
// The reference recurses per sample: castRay -> shade surface = emission (camera rays or non-light
// objects) + direct light + traced specular (and glossy) reflection / transmission, up to
// maxRayGeneration. Here the recursion is a wavefront of tasks (ray, sample slot, weight,
// generation, high-quality flag, branch key); per generation:
//   trace tasks (closest) -> shade: emission into the sample, shadow rays of the direct term into a
//   shadow queue (each with its finished contribution), children into the next task queue ->
//   trace shadow rays (any hit) -> add the unoccluded contributions -> next generation.
// High-quality vertices (camera rays and specular chains) estimate every light with its
// numberOfEmissionSamples light samples and as many BSDF samples, combined with the squared (power)
// heuristic on sample-count-weighted densities; glossy children are low quality: one light chosen
// by power per numberOfSecondaryLightSamples. The reference draws high-quality vertices' samples
// from per-sample subsequences shared by all generations and low-quality ones from a secondary
// random stream; here the former are stratified sampler dimensions fixed per light and sample, the
// latter hashes of a per-task branch key.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/liar_gpu.h"
#include "ctx.h"
#include "photon_mapper.h"
#include "render_dev.cuh"

using namespace liar_gpu;
using namespace liar_gpu::rt;

namespace liar_gpu {
namespace rt {
const DScene& scene_dscene(const liar_gpu_scene* s);
const liar_gpu_mesh* scene_mesh(const liar_gpu_scene* s);
const std::vector<liar_light>& scene_lights(const liar_gpu_scene* s);
const std::vector<liar_material>& scene_materials(const liar_gpu_scene* s);
unsigned long long* render_stats_device(liar_gpu_ctx* ctx, cudaStream_t st);
}  // namespace rt
}  // namespace liar_gpu

namespace {

// shadow rays end this fraction short of the light's surface, so that the light's own triangles
// are never taken for occluders at float precision
constexpr float kShadowShrink = 1e-4f;

struct DTasks {
    liar_ray* rays;
    uint32_t* slot;
    float* T;
    uint32_t* meta;  // generation (bits 0-7), high quality (bit 8)
    uint32_t* key;   // branch key of the task tree (low-quality sample streams)
    uint32_t* count;
};

struct DShadows {
    liar_ray* rays;
    uint32_t* slot;
    float* value;
    uint32_t* count;
};

struct DSamples {
    float* lam;
    float* lam_pdf;
    float* L;
    float* alpha;
};

struct DParams {
    liar_camera cam;
    int width, height, spp, max_gen;
    uint64_t seed;
    uint64_t first_path;
    int n_secondary;
    uint32_t glossy;  // CAP_GLOSSY when glossy reflection/transmission is traced
    unsigned long long* stats;
    FilmSpec film;
    // PhotonMapper (photon_mapper.cpp:466-518): 0 off, 1 render, 2 visualise the photon map;
    // vertices that estimate from the maps append their hit point and task index here
    int pm;
    int pm_direct;       // isRayTracingDirect
    float* q_pos;
    uint32_t* q_task;
    uint32_t* q_count;
};

// sampler dimensions (disjoint from the path tracer's and from each other)
__host__ __device__ __forceinline__ uint32_t dim_light(int l, int k, int axis) {  // axis 0,1 light 2D; 2,3 BSDF 2D; 4 component
    return 0x200000u + ((uint32_t)l * 1024u + (uint32_t)k) * 8u + (uint32_t)axis;
}
__host__ __device__ __forceinline__ uint32_t dim_scatter(int i, int axis) {  // 0,1,2 reflection; 3,4,5 transmission
    return 0x400000u + (uint32_t)i * 8u + (uint32_t)axis;
}
__host__ __device__ __forceinline__ uint32_t dim_branch(uint32_t key, uint32_t j) {
    return 0x80000000u | (uint32_t)(mix64(((uint64_t)key << 20) ^ j) & 0x7fffffffu);
}
__host__ __device__ __forceinline__ uint32_t child_key(uint32_t key, uint32_t c) {
    return (uint32_t)mix64(((uint64_t)key << 8) | (c + 1u)) | 1u;
}

__device__ __forceinline__ SampleKey dkey(const DParams& W, uint64_t g) {
    SampleKey k;
    k.seed = W.seed;
    k.pixel = (uint32_t)(g / (uint64_t)W.spp);
    k.sample = (uint32_t)(g % (uint64_t)W.spp);
    k.spp = (uint32_t)W.spp;
    return k;
}

// warp-aggregated appends of a per-lane count: returns the lane's first index
__device__ __forceinline__ uint32_t warp_reserve(uint32_t* counter, uint32_t n) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t incl = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += v;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    uint32_t base = 0;
    if (lane == 31 && total) base = atomicAdd(counter, total);
    base = __shfl_sync(0xffffffffu, base, 31);
    return base + incl - n;
}

__device__ __forceinline__ void put_ray(liar_ray* rays, uint32_t i, float3 o, float3 d, float tmin, float tmax) {
    float4* dst = reinterpret_cast<float4*>(rays + i);
    dst[0] = make_float4(o.x, o.y, o.z, tmin);
    dst[1] = make_float4(d.x, d.y, d.z, tmax);
}

// a reserved entry that turned out unused: a ray with a NaN origin, which the trace kernel
// retires without touching the tree
__device__ __forceinline__ void put_void_ray(liar_ray* rays, uint32_t i) {
    const float nan = __int_as_float(0x7fffffff);
    float4* dst = reinterpret_cast<float4*>(rays + i);
    dst[0] = make_float4(nan, nan, nan, 0.0f);
    dst[1] = make_float4(0.0f, 0.0f, 1.0f, 0.0f);
}

__global__ void __launch_bounds__(256) k_dl_raygen(DScene S, DParams W, DSamples P, DTasks out, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const SampleKey k = dkey(W, W.first_path + i);
    float lpdf;
    const float lam = observer_sample(S, sample_dim(k, DIM_LAMBDA, true), lpdf);
    const liar_ray r = camera_ray(W.cam, k, W.width, W.height);
    P.lam[i] = lam;
    P.lam_pdf[i] = lpdf;
    P.L[i] = 0.0f;
    P.alpha[i] = 0.0f;
    reinterpret_cast<float4*>(out.rays + i)[0] = make_float4(r.ox, r.oy, r.oz, r.tmin);
    reinterpret_cast<float4*>(out.rays + i)[1] = make_float4(r.dx, r.dy, r.dz, r.tmax);
    out.slot[i] = i;
    out.T[i] = 1.0f;
    out.meta[i] = 0u | (1u << 8);
    out.key[i] = 1u;
    if (i == 0) *out.count = n;
}

// the shadow rays of one task: `reserved` entries from `base`, filled in order, the rest voided
struct ShadowWriter {
    DShadows q;
    uint32_t base, j, reserved;
    __device__ void put(float3 o, float3 d, float tmax, uint32_t slot, float value) {
        if (j >= reserved) return;
        const uint32_t i = base + j++;
        put_ray(q.rays, i, o, d, kTol, tmax);
        q.slot[i] = slot;
        q.value[i] = value;
    }
    __device__ void finish(uint32_t slot) {
        while (j < reserved) {
            const uint32_t i = base + j++;
            put_void_ray(q.rays, i);
            q.slot[i] = slot;
            q.value[i] = 0.0f;
        }
    }
};

// RayTracer::estimateLightContribution for light l with nl light and nb BSDF samples; u(kind, k, axis)
// gives the sample values
template <class U>
__device__ void estimate_light(const DScene& S, const Bsdf& B, const HitContext& HC, float3 wi, float3 start, int l,
                               int nl, int nb, float lam, float scale, uint32_t slot, ShadowWriter& out, const U& u) {
    const liar_light L = S.lights[l];
    const bool singular = L.type == LIAR_LIGHT_POINT;
    uint32_t caps = CAP_REFL | CAP_TRANS | CAP_DIFF | CAP_GLOSSY;
    if (!singular) caps |= CAP_SPEC;
    const float fnl = (float)nl, fnb = (float)nb;
    for (int k = 0; k < nl; ++k) {
        const LightSample ls = light_sample(S, l, start, u(0, k, 0), u(0, k, 1), lam);
        if (ls.pdf <= 0.0f || ls.value == 0.0f) continue;
        // LightArea::doSampleEmission with the target normal: lights behind the surface give nothing
        if ((L.type == LIAR_LIGHT_AREA_PARALLELOGRAM || L.type == LIAR_LIGHT_AREA_MESH) && dot(HC.N, ls.dir) <= 0.0f)
            continue;
        const float3 wo = mk(dot(ls.dir, HC.u), dot(ls.dir, HC.v), dot(ls.dir, HC.N));
        const BsdfOut be = bsdf_evaluate(B, wi, wo, caps);
        if (be.value == 0.0f || !(be.pdf > 0.0f)) continue;
        const float w = power_heuristic(fnl * ls.pdf, fnb * be.pdf);
        const float v = scale * be.value * ls.value * (w * fabsf(wo.z) / (fnl * ls.pdf));
        out.put(start, ls.dir, ls.dist * (1.0f - kShadowShrink), slot, v);
    }
    const bool specular = B.type == LIAR_MAT_MIRROR || B.type == LIAR_MAT_CONDUCTOR || B.type == LIAR_MAT_DIELECTRIC;
    for (int k = 0; k < nb; ++k) {
        const BsdfSample bs = bsdf_sample(B, wi, u(1, k, 0), u(1, k, 1), u(2, k, 0), caps);
        if (!bs.ok()) continue;
        const float3 wd = bs.wo.x * HC.u + bs.wo.y * HC.v + bs.wo.z * HC.N;
        const LightEmission e = light_emission(S, l, start, wd, lam);
        if (!(e.pdf > 0.0f) || e.value == 0.0f) continue;
        const float w = specular ? 1.0f : power_heuristic(fnb * bs.pdf, fnl * e.pdf);
        const float v = scale * bs.value * e.value * (w * fabsf(bs.wo.z) / (fnb * bs.pdf));
        out.put(start, wd, e.t * (1.0f - kShadowShrink), slot, v);
    }
}

__global__ void __launch_bounds__(128) k_dl_shade(DScene S, DParams W, DSamples P, DTasks in,
                                                  const liar_hit* __restrict__ hits, uint32_t n_in, DTasks out,
                                                  DShadows sh, uint32_t shadow_hq) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = q < n_in;
    uint32_t p = 0, meta = 0, key = 0;
    float T = 0.0f;
    float4 r0 = make_float4(0, 0, 0, 0), r1 = make_float4(0, 0, 1, 0);
    liar_hit h{-1, 0.0f};
    if (valid) {
        p = in.slot[q];
        T = in.T[q];
        meta = in.meta[q];
        key = in.key[q];
        r0 = reinterpret_cast<const float4*>(in.rays + q)[0];
        r1 = reinterpret_cast<const float4*>(in.rays + q)[1];
        h = hits[q];
    }
    const int gen = (int)(meta & 0xffu);
    const bool hq = (meta >> 8) & 1u;
    const bool shading = valid && h.prim >= 0 && gen <= W.max_gen;
    const bool more = gen + 1 <= W.max_gen;
    const float3 o = mk(r0.x, r0.y, r0.z), d = mk(r1.x, r1.y, r1.z);
    HitContext HC;
    HC.mat = -1;
    HC.light = -1;
    liar_material M{};
    Bsdf B{};
    bool has_bsdf = false;
    float lam = 0.0f;
    // the exact numbers of shadow rays and children this task writes (failed samples are voided)
    uint32_t n_sh = 0, n_ch = 0;
    const uint32_t sg = CAP_REFL | CAP_TRANS | CAP_SPEC | W.glossy;
    if (shading) {
        HC = hit_context(S, o, d, (uint32_t)h.prim);
        if (HC.mat < 0) {
            n_ch = more ? 1u : 0u;  // no shader: continue through the surface
        } else {
            M = S.mats[HC.mat];
            lam = P.lam[p];
            if (M.type != LIAR_MAT_NONE) {
                B = make_bsdf(S, M, HC, lam);
                has_bsdf = true;
                n_sh = hq ? shadow_hq : (S.n_lights > 0 ? 2u * (uint32_t)W.n_secondary : 0u);
                if (W.pm == 2 || (W.pm == 1 && !W.pm_direct)) n_sh = 0u;  // no traced direct light
                if (compatible_caps(B.caps, sg) && more && W.pm != 2) {
                    const uint32_t ns = hq ? (uint32_t)(M.samples > 0 ? M.samples : 1) : 1u;
                    n_ch = (has_caps(B.caps, CAP_REFL) ? ns : 0u) + (has_caps(B.caps, CAP_TRANS) ? ns : 0u);
                }
            }
        }
    }
    // PhotonMapper: vertices with a shader query the photon maps (the visualisation), or those with
    // a diffuse component do (estimateCaustics, estimateRadiance)
    const bool query = W.pm != 0 && shading && HC.mat >= 0 &&
                       (W.pm == 2 || (has_bsdf && has_caps(B.caps, CAP_DIFF)));
    if (W.pm != 0) {  // uniform over the launch: every lane of the warp takes the reservation
        const uint32_t qi = warp_reserve(W.q_count, query ? 1u : 0u);
        if (query) {
            W.q_pos[3 * (size_t)qi] = HC.target.x;
            W.q_pos[3 * (size_t)qi + 1] = HC.target.y;
            W.q_pos[3 * (size_t)qi + 2] = HC.target.z;
            W.q_task[qi] = q;
        }
    }
    ShadowWriter sw{sh, warp_reserve(sh.count, n_sh), 0u, n_sh};
    const uint32_t cbase = warp_reserve(out.count, n_ch);
    uint32_t nc = 0;
    auto child = [&](float3 co, float3 cd, float tmin, float tmax, float Tc, bool hq_c, uint32_t c) {
        if (nc >= n_ch) return;
        const uint32_t i = cbase + nc++;
        put_ray(out.rays, i, co, cd, tmin, tmax);
        out.slot[i] = p;
        out.T[i] = Tc;
        out.meta[i] = (uint32_t)(gen + 1) | (hq_c ? (1u << 8) : 0u);
        out.key[i] = child_key(key, c);
    };
    if (valid && h.prim < 0) {
        // the sky is an object without a shader: the camera ray sees it (alpha), nothing more
        if (gen == 0 && S.sky_light >= 0 && S.sky_distance > r0.w * (1.0f + kTol) && S.sky_distance < r1.w * (1.0f - kTol))
            P.alpha[p] = 1.0f;
    }
    if (shading) {
        if (gen == 0) P.alpha[p] = 1.0f;
        if (HC.mat < 0) {
            child(o, d, h.t + kTol, r1.w, T, hq, 0);
        } else {
            const SampleKey skey = dkey(W, W.first_path + p);
            // shader emission: camera rays see light objects, other emitters are always seen
            if (W.pm != 2 && (gen == 0 || HC.light < 0) && M.emission >= 0)
                atomicAdd(&P.L[p], T * spec_eval(S, M.emission, lam, false));
            if (has_bsdf && W.pm != 2) {
                const float3 md = -d;
                float3 wi = mk(dot(md, HC.u), dot(md, HC.v), dot(md, HC.N));
                wi.z = fmaxf(wi.z, kEps);
                const float3 start = HC.target + (10.0f * kTol) * HC.N;
                // ---- direct light (traceDirect)
                if (W.pm == 1 && !W.pm_direct) {
                    // the PhotonMapper without traced direct light: the global map holds it
                } else if (hq) {
                    for (int l = 0; l < S.n_lights; ++l) {
                        const liar_light& L = S.lights[l];
                        const int nl = L.emission_samples > 0 ? L.emission_samples : 1;
                        const int nb = L.type == LIAR_LIGHT_POINT ? 0 : nl;
                        auto u = [&](int kind, int k, int axis) {
                            const int ax = kind == 0 ? axis : (kind == 1 ? 2 + axis : 4);
                            return sample_dim(skey, dim_light(l, k, ax), true);
                        };
                        estimate_light(S, B, HC, wi, start, l, nl, nb, lam, T, p, sw, u);
                    }
                } else if (S.n_lights > 0) {
                    const int n = W.n_secondary;
                    for (int k = 0; k < n; ++k) {
                        const uint32_t j0 = 16u * (uint32_t)k;
                        const float uc = sample_dim(skey, dim_branch(key, j0), false);
                        int l = lower_bound_f(S.light_cdf, S.n_lights, uc);
                        if (l > S.n_lights - 1) l = S.n_lights - 1;
                        const float pc = light_choice_pdf(S, l);
                        if (!(pc > 0.0f)) continue;
                        const int nb = S.lights[l].type == LIAR_LIGHT_POINT ? 0 : 1;
                        auto u = [&](int kind, int, int axis) {
                            return sample_dim(skey, dim_branch(key, j0 + 1u + 2u * (uint32_t)kind + (uint32_t)axis), false);
                        };
                        estimate_light(S, B, HC, wi, start, l, 1, nb, lam, T / ((float)n * pc), p, sw, u);
                    }
                }
                // ---- traced specular and glossy scattering (traceSpecularAndGlossy)
                if (n_ch > 0) {
                    const bool specular =
                        B.type == LIAR_MAT_MIRROR || B.type == LIAR_MAT_CONDUCTOR || B.type == LIAR_MAT_DIELECTRIC;
                    const int ns = hq ? (M.samples > 0 ? M.samples : 1) : 1;
                    for (int side = 0; side < 2; ++side) {
                        const uint32_t dir_cap = side == 0 ? CAP_REFL : CAP_TRANS;
                        if (!has_caps(B.caps, dir_cap)) continue;
                        for (int i = 0; i < ns; ++i) {
                            float u0, u1, uc;
                            if (hq) {
                                u0 = sample_dim(skey, dim_scatter(i, 3 * side), true);
                                u1 = sample_dim(skey, dim_scatter(i, 3 * side + 1), true);
                                uc = sample_dim(skey, dim_scatter(i, 3 * side + 2), true);
                            } else {
                                const uint32_t j0 = 0x1000u + 8u * (uint32_t)side;
                                u0 = sample_dim(skey, dim_branch(key, j0), false);
                                u1 = sample_dim(skey, dim_branch(key, j0 + 1u), false);
                                uc = sample_dim(skey, dim_branch(key, j0 + 2u), false);
                            }
                            const BsdfSample bs = bsdf_sample(B, wi, u0, u1, uc, dir_cap | CAP_SPEC | W.glossy);
                            if (!bs.ok() || (side == 0 ? !(bs.wo.z > 0.0f) : !(bs.wo.z < 0.0f))) continue;
                            const float3 wd = bs.wo.x * HC.u + bs.wo.y * HC.v + bs.wo.z * HC.N;
                            const float3 begin = HC.target + ((side == 0 ? 10.0f : -10.0f) * kTol) * HC.N;
                            const float Tc = T * bs.value * (fabsf(bs.wo.z) / ((float)ns * bs.pdf));
                            child(begin, wd, kTol, INFINITY, Tc, hq && specular, 2u * (uint32_t)i + (uint32_t)side);
                        }
                    }
                }
            }
        }
    }
    sw.finish(p);
    while (nc < n_ch) {  // children whose sample failed: void tasks
        const uint32_t i = cbase + nc++;
        put_void_ray(out.rays, i);
        out.slot[i] = p;
        out.T[i] = 0.0f;
        out.meta[i] = (uint32_t)(W.max_gen + 1);
        out.key[i] = 0u;
    }
    const uint32_t lane = threadIdx.x & 31u;
    unsigned long long segs = valid ? 1ull : 0ull, n_hit = (valid && h.prim >= 0) ? 1ull : 0ull;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        segs += __shfl_down_sync(0xffffffffu, segs, off);
        n_hit += __shfl_down_sync(0xffffffffu, n_hit, off);
    }
    if (lane == 0 && segs) {
        atomicAdd(W.stats + 1, segs);
        atomicAdd(W.stats + 2, n_hit);
    }
}

__global__ void k_dl_shadow_add(DShadows sh, uint32_t n, const liar_hit* __restrict__ hits, float* L) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = sh.value[i];
    if (v != 0.0f && hits[i].prim < 0) atomicAdd(&L[sh.slot[i]], v);
}

// ---- PhotonMapper estimates at the queried vertices (photon_mapper.cpp:1282-1381, 1254-1279)
enum { kEstRadiance = 0, kEstCaustics = 1, kEstIrradiance = 2 };

// Photon::spectralPower: the XYZ power as a spectrum at the sample's wavelength (Spectral::fromXYZ,
// an illuminant), through the photon's precomputed blend
__device__ __forceinline__ float photon_power(const PmMap& M, const DRecovery& R, int32_t i, float lam) {
    RecoveryBlend b;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        b.idx[j] = M.blend_idx[3 * (size_t)i + j];
        b.w[j] = M.blend_w[3 * (size_t)i + j];
    }
    return recovery_eval(R, b, lam, false);
}

// one thread per queried vertex: the vertex's BSDF against the k nearest photons of one map
//   kEstRadiance:   sum f(w, w_p) Phi_p(lam) / (pi r^2), f without its specular and glossy parts,
//                   at least two photons (estimateRadiance without an irradiance map)
//   kEstCaustics:   the same with the Gaussian filter w = alpha (1 - (1 - e^(-beta d^2 / 2r^2)) /
//                   (1 - e^-beta)), alpha 0.918, beta 1.953, f's diffuse part (estimateCaustics)
//   kEstIrradiance: the XYZ of the photons arriving from the normal's side over pi r^2, as a
//                   spectrum at lam (isVisualizingPhotonMap: estimateIrradianceImpl)
// r^2 is the squared distance of the farthest photon found; the result, times the task's weight,
// is added to the sample's radiance
__global__ void __launch_bounds__(128) k_pm_estimate(DScene S, DParams W, DSamples P, DTasks tin,
                                                     const liar_hit* __restrict__ hits, const uint32_t* __restrict__ q_task,
                                                     uint32_t n_q, PmMap M, DRecovery R, int kind,
                                                     const int32_t* __restrict__ g_idx, const float* __restrict__ g_d2,
                                                     const int32_t* __restrict__ g_cnt) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_q) return;
    const int k = M.k;
    const int cnt = min(g_cnt[i], k);
    if (cnt < (kind == kEstIrradiance ? 1 : 2)) return;
    const uint32_t q = q_task[i];
    const uint32_t p = tin.slot[q];
    const float T = tin.T[q];
    const float4 r0 = reinterpret_cast<const float4*>(tin.rays + q)[0];
    const float4 r1 = reinterpret_cast<const float4*>(tin.rays + q)[1];
    const float3 d = mk(r1.x, r1.y, r1.z);
    const HitContext HC = hit_context(S, mk(r0.x, r0.y, r0.z), d, (uint32_t)hits[q].prim);
    const float lam = P.lam[p];
    const int32_t* idx = g_idx + (size_t)i * k;
    const float r2 = g_d2[(size_t)i * k + cnt - 1];
    if (!(r2 > 0.0f)) return;
    float result = 0.0f;
    if (kind == kEstIrradiance) {
        float X = 0.0f, Y = 0.0f, Z = 0.0f;
        for (int j = 0; j < cnt; ++j) {
            const int32_t ph = idx[j];
            if (ph < 0 || (uint64_t)ph >= M.n) continue;
            if (M.omega_in[3 * (size_t)ph] * HC.N.x + M.omega_in[3 * (size_t)ph + 1] * HC.N.y +
                    M.omega_in[3 * (size_t)ph + 2] * HC.N.z > 0.0f) {
                X += M.power[3 * (size_t)ph];
                Y += M.power[3 * (size_t)ph + 1];
                Z += M.power[3 * (size_t)ph + 2];
            }
        }
        const float inv = 1.0f / (3.14159265358979323846f * r2);
        RecoveryBlend b;
        if (recovery_locate(R, X * inv, Y * inv, Z * inv, b)) result = recovery_eval(R, b, lam, false);
    } else {
        const liar_material Mat = S.mats[HC.mat];
        const Bsdf B = make_bsdf(S, Mat, HC, lam);
        const float3 md = -d;
        float3 wi = mk(dot(md, HC.u), dot(md, HC.v), dot(md, HC.N));
        wi.z = fmaxf(wi.z, kEps);
        const uint32_t caps = kind == kEstRadiance ? (CAP_ALL & ~CAP_SPEC & ~CAP_GLOSSY) : (CAP_REFL | CAP_TRANS | CAP_DIFF);
        const float alpha = 0.918f, beta = 1.953f;
        const float b1 = -beta / (2.0f * r2), b2 = 1.0f / (1.0f - expf(-beta));
        for (int j = 0; j < cnt; ++j) {
            const int32_t ph = idx[j];
            if (ph < 0 || (uint64_t)ph >= M.n) continue;
            const float3 om = mk(M.omega_in[3 * (size_t)ph], M.omega_in[3 * (size_t)ph + 1], M.omega_in[3 * (size_t)ph + 2]);
            const float3 wo = mk(dot(om, HC.u), dot(om, HC.v), dot(om, HC.N));
            const BsdfOut be = bsdf_evaluate(B, wi, wo, caps);
            if (!(be.pdf > 0.0f) || be.value == 0.0f) continue;
            float v = be.value * photon_power(M, R, ph, lam);
            if (kind == kEstCaustics) v *= alpha * (1.0f - b2 * (1.0f - expf(b1 * g_d2[(size_t)i * k + j])));
            result += v;
        }
        result /= 3.14159265358979323846f * r2;
    }
    if (result != 0.0f) atomicAdd(&P.L[p], T * result);
}

__global__ void k_dl_splat(DScene S, DParams W, DSamples P, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float lam_pdf = P.lam_pdf[i], L = P.L[i];
    float3 xyz = mk(0, 0, 0);
    if (lam_pdf > 0.0f) {
        const float s = L / lam_pdf;
        const float3 c = observer_sensitivity(S, P.lam[i]);
        xyz = mk(s * c.x, s * c.y, s * c.z);
    }
    film_splat(W.film, dkey(W, W.first_path + i), xyz, P.alpha[i]);
}

struct DirectBuffers {
    size_t n_samples = 0, n_tasks[2] = {0, 0}, n_shadows = 0;
    void* samples = nullptr;
    void* tasks[2] = {nullptr, nullptr};
    void* shadows = nullptr;
    liar_hit* hits = nullptr;
    size_t hits_cap = 0;
    uint32_t* counters = nullptr;  // [0] task count A, [1] task count B, [2] shadow count, [3] map queries
    uint32_t* h_counters = nullptr;
    // PhotonMapper: the queried vertices (3 floats, a task index and a gather count each) and one
    // map's gather results (k indices and squared distances per vertex)
    void* queries = nullptr;
    size_t n_queries = 0;
    void* gathers = nullptr;
    size_t n_gathers = 0;
};

DirectBuffers* direct_buffers(liar_gpu_ctx* ctx) {
    for (auto& ext : ctx->extensions)
        if (ext.first == "direct") return static_cast<DirectBuffers*>(ext.second);
    DirectBuffers* b = new DirectBuffers();
    ctx->extensions.emplace_back("direct", b);
    ctx->on_destroy.push_back([b]() {
        for (void* p : {b->samples, b->tasks[0], b->tasks[1], b->shadows, (void*)b->hits, (void*)b->counters, b->queries,
                        b->gathers})
            if (p) cudaFree(p);
        if (b->h_counters) cudaFreeHost(b->h_counters);
        delete b;
    });
    return b;
}

int grow(liar_gpu_ctx* ctx, void** p, size_t* cap, size_t want, size_t unit, const char* what) {
    if (*cap >= want) return LIAR_OK;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    const size_t n = want + want / 4 + 1024;
    cudaError_t e = cudaMalloc(p, n * unit);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return ctx_cuda(ctx, e, what);
    }
    *cap = n;
    return LIAR_OK;
}

DTasks task_view(void* base, size_t cap, uint32_t* count) {
    char* c = static_cast<char*>(base);
    DTasks t;
    t.rays = reinterpret_cast<liar_ray*>(c);
    t.slot = reinterpret_cast<uint32_t*>(c + cap * 32);
    t.T = reinterpret_cast<float*>(c + cap * 36);
    t.meta = reinterpret_cast<uint32_t*>(c + cap * 40);
    t.key = reinterpret_cast<uint32_t*>(c + cap * 44);
    t.count = count;
    return t;
}

}  // namespace

namespace liar_gpu {
namespace rt {

int render_direct(liar_gpu_ctx* ctx, const liar_gpu_scene* scene, const liar_render_desc& R, float* d_film,
                  cudaStream_t st, const PmMaps* pm) {
    if (R.max_ray_generation < 0 || R.max_ray_generation > 250)
        return ctx_fail(ctx, LIAR_ERR_INVALID, "max_ray_generation must lie in [0, 250]");
    const uint64_t total = (uint64_t)R.width * R.height * R.spp;
    if ((uint64_t)R.width * R.height >= (1ull << 32)) return ctx_fail(ctx, LIAR_ERR_INVALID, "image too large");
    const std::vector<liar_light>& lights = scene_lights(scene);
    const std::vector<liar_material>& mats = scene_materials(scene);
    const int n_sec = R.secondary_light_samples > 0 ? R.secondary_light_samples : 1;
    // worst cases per task: shadow rays of the direct term and children
    uint64_t sh_hq = 0;
    for (const liar_light& L : lights) {
        const uint64_t nl = L.emission_samples > 0 ? (uint64_t)L.emission_samples : 1;
        if (nl > 1024) return ctx_fail(ctx, LIAR_ERR_UNSUPPORTED, "at most 1024 emission samples per light");
        sh_hq += nl + (L.type == LIAR_LIGHT_POINT ? 0 : nl);
    }
    const uint64_t sh_lq = lights.empty() ? 0 : 2ull * (uint64_t)n_sec;
    const uint32_t shadow_per_task = (uint32_t)std::max<uint64_t>(std::max(sh_hq, sh_lq), 1);
    uint32_t children = 1;  // continue-through
    for (const liar_material& M : mats) {
        const uint32_t ns = M.samples > 0 ? (uint32_t)M.samples : 1;
        if (ns > 64) return ctx_fail(ctx, LIAR_ERR_UNSUPPORTED, "at most 64 reflection samples per shader");
        children = std::max(children, 2 * ns);
    }
    // samples per wave: keep the first generation's shadow queue near 1 GiB
    uint64_t wave = R.wave_paths > 0 ? (uint64_t)R.wave_paths
                                     : std::max<uint64_t>(4096, (1ull << 30) / (40ull * shadow_per_task + 64));
    wave = std::min<uint64_t>(std::min<uint64_t>(wave, total), 1ull << 22);
    DirectBuffers* b = direct_buffers(ctx);
    int rc = LIAR_OK;
    if (!b->counters) {
        cudaError_t e = cudaMalloc((void**)&b->counters, 16 * sizeof(uint32_t));
        if (e == cudaSuccess) e = cudaMallocHost((void**)&b->h_counters, 16 * sizeof(uint32_t));
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "direct lighting counters");
    }
    rc = grow(ctx, &b->samples, &b->n_samples, wave, 16, "direct lighting samples");
    if (rc) return rc;
    unsigned long long* stats = render_stats_device(ctx, st);
    if (!stats) return ctx_fail(ctx, LIAR_ERR_OOM, "render statistics");
    cudaError_t e = cudaMemsetAsync(stats, 0, 4 * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "reset statistics");
    DParams W;
    W.cam = R.camera;
    W.width = R.width;
    W.height = R.height;
    W.spp = R.spp;
    W.film = film_spec(d_film, R);
    W.max_gen = R.max_ray_generation;
    W.seed = mix64(R.seed ^ mix64(0x51ed270b27ad0e0dull + (uint64_t)(uint32_t)R.first_sample));
    W.n_secondary = n_sec;
    W.glossy = R.trace_glossy < 0 ? 0u : CAP_GLOSSY;
    W.stats = stats;
    W.pm = pm ? (pm->visualize ? 2 : 1) : 0;
    W.pm_direct = pm ? pm->ray_direct : 1;
    W.q_pos = nullptr;
    W.q_task = nullptr;
    W.q_count = b->counters + 3;
    const DScene& S = scene_dscene(scene);
    const liar_gpu_mesh* mesh = scene_mesh(scene);
    for (uint64_t first = 0; first < total; first += wave) {
        const uint32_t n = (uint32_t)std::min<uint64_t>(wave, total - first);
        DSamples P;
        P.lam = static_cast<float*>(b->samples);
        P.lam_pdf = P.lam + b->n_samples;
        P.L = P.lam_pdf + b->n_samples;
        P.alpha = P.L + b->n_samples;
        W.first_path = first;
        rc = grow(ctx, &b->tasks[0], &b->n_tasks[0], n, 48, "direct lighting tasks");
        if (rc) return rc;
        e = cudaMemsetAsync(b->counters, 0, 16 * sizeof(uint32_t), st);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "reset counters");
        k_dl_raygen<<<(n + 255) / 256, 256, 0, st>>>(S, W, P, task_view(b->tasks[0], b->n_tasks[0], b->counters), n);
        uint32_t n_in = n;
        int cur = 0;
        for (int gen = 0; n_in > 0 && gen <= W.max_gen; ++gen) {
            // the next generation's queue and this generation's shadow rays at their worst case
            const uint64_t want_children = gen + 1 <= W.max_gen ? (uint64_t)n_in * children : 0;
            const uint64_t want_shadows = (uint64_t)n_in * shadow_per_task;
            if (want_children > (1ull << 31) || want_shadows > (1ull << 31))
                return ctx_fail(ctx, LIAR_ERR_UNSUPPORTED,
                                "direct lighting wave too large for its task tree: set render.wave_paths lower");
            // (the other task queue holds nothing live: the host waited for the previous generation)
            rc = grow(ctx, &b->tasks[cur ^ 1], &b->n_tasks[cur ^ 1], std::max<uint64_t>(want_children, 1), 48,
                      "direct lighting tasks");
            if (!rc) rc = grow(ctx, &b->shadows, &b->n_shadows, std::max<uint64_t>(want_shadows, 1), 40,
                               "direct lighting shadows");
            if (!rc && b->hits_cap < std::max<uint64_t>(std::max<uint64_t>(want_shadows, n_in), 1)) {
                void* hp = b->hits;
                rc = grow(ctx, &hp, &b->hits_cap, std::max<uint64_t>(want_shadows, n_in), 8, "direct lighting hits");
                b->hits = static_cast<liar_hit*>(hp);
            }
            if (!rc && pm) {
                rc = grow(ctx, &b->queries, &b->n_queries, n_in, 20, "photon map queries");
                W.q_pos = static_cast<float*>(b->queries);
                W.q_task = reinterpret_cast<uint32_t*>(static_cast<char*>(b->queries) + b->n_queries * 12);
            }
            if (rc) return rc;
            const DTasks tin = task_view(b->tasks[cur], b->n_tasks[cur], b->counters + cur);
            const DTasks tout = task_view(b->tasks[cur ^ 1], b->n_tasks[cur ^ 1], b->counters + (cur ^ 1));
            DShadows sq;
            char* sc = static_cast<char*>(b->shadows);
            sq.rays = reinterpret_cast<liar_ray*>(sc);
            sq.slot = reinterpret_cast<uint32_t*>(sc + b->n_shadows * 32);
            sq.value = reinterpret_cast<float*>(sc + b->n_shadows * 36);
            sq.count = b->counters + 2;
            rc = trace_mesh_internal(ctx, mesh, tin.rays, n_in, b->hits, 0, st, kCounterWord + 10);
            if (rc) return rc;
            e = cudaMemsetAsync(b->counters + (cur ^ 1), 0, 4, st);
            if (e == cudaSuccess) e = cudaMemsetAsync(b->counters + 2, 0, 8, st);
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "reset queues");
            k_dl_shade<<<(n_in + 127) / 128, 128, 0, st>>>(S, W, P, tin, b->hits, n_in, tout, sq, (uint32_t)sh_hq);
            e = cudaGetLastError();
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "direct lighting shade launch");
            e = cudaMemcpyAsync(b->h_counters, b->counters, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "direct lighting queue sizes");
            const uint32_t n_sh = b->h_counters[2];
            if ((uint64_t)n_sh > want_shadows || (uint64_t)b->h_counters[cur ^ 1] > want_children)
                return ctx_fail(ctx, LIAR_ERR_INVALID, "direct lighting queue overflow");
            // the photon-map estimates of the queried vertices, while the tasks' hits are current
            const uint32_t n_q = pm ? b->h_counters[3] : 0u;
            if (n_q > n_in) return ctx_fail(ctx, LIAR_ERR_INVALID, "photon map query overflow");
            for (int m = 0; n_q > 0 && m < 2; ++m) {
                const PmMap& M = pm->map[m];
                if (pm->visualize && m != kPmGlobal) continue;
                if (M.n == 0 || M.k < 1 || !M.grid) continue;
                rc = grow(ctx, &b->gathers, &b->n_gathers, (size_t)n_q * M.k, 8, "photon gathers");
                if (rc) return rc;
                int32_t* g_idx = static_cast<int32_t*>(b->gathers);
                float* g_d2 = reinterpret_cast<float*>(g_idx + b->n_gathers);
                int32_t* g_cnt = reinterpret_cast<int32_t*>(b->queries) + 4 * b->n_queries;  // after positions and tasks
                rc = liar_gpu_photon_gather_device(ctx, M.grid, W.q_pos, n_q, M.k, g_idx, g_d2, g_cnt, st);
                if (rc) return rc;
                const int kind = pm->visualize ? kEstIrradiance : (m == kPmGlobal ? kEstRadiance : kEstCaustics);
                k_pm_estimate<<<(n_q + 127) / 128, 128, 0, st>>>(S, W, P, tin, b->hits, W.q_task, n_q, M, pm->rec, kind,
                                                                  g_idx, g_d2, g_cnt);
                e = cudaGetLastError();
                if (e != cudaSuccess) return ctx_cuda(ctx, e, "photon estimate launch");
            }
            if (n_sh > 0) {
                rc = trace_mesh_internal(ctx, mesh, sq.rays, n_sh, b->hits, 1, st, kCounterWord + 10);
                if (rc) return rc;
                k_dl_shadow_add<<<(n_sh + 255) / 256, 256, 0, st>>>(sq, n_sh, b->hits, P.L);
                e = cudaGetLastError();
                if (e != cudaSuccess) return ctx_cuda(ctx, e, "direct lighting shadow launch");
            }
            cur ^= 1;
            n_in = b->h_counters[cur];
        }
        k_dl_splat<<<(n + 255) / 256, 256, 0, st>>>(S, W, P, n);
        e = cudaGetLastError();
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "direct lighting splat");
    }
    unsigned long long paths = total;
    e = cudaMemcpyAsync(stats, &paths, sizeof(paths), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "direct lighting statistics");
    return ctx_check_status(ctx);
}

}  // namespace rt
}  // namespace liar_gpu
