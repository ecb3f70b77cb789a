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
    uint32_t sampler;  // SAMPLER_* mode bits (sampler.h)
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
    uint32_t* q_task;    // bit 31: the vertex gathers its indirect light (no radiance estimate)
    uint32_t* q_count;
    int fg_rays;         // final gathering: rays per high-quality diffuse vertex (0: none)
    int fg_secondary;    // numSecondaryGatherRays
    DTasks fg;           // the gather rays of this generation (meta: stage in bit 9)
};

constexpr uint32_t kNoRadiance = 0x80000000u;
constexpr uint32_t kStage1 = 1u << 9;

// sampler dimensions (disjoint from the path tracer's and from each other)
__host__ __device__ __forceinline__ uint32_t dim_light(int l, int k, int axis) {  // axis 0,1 light 2D; 2,3 BSDF 2D; 4 component
    return 0x200000u + ((uint32_t)l * 1024u + (uint32_t)k) * 8u + (uint32_t)axis;
}
__host__ __device__ __forceinline__ uint32_t dim_scatter(int i, int axis) {  // 0,1,2 reflection; 3,4,5 transmission
    return 0x400000u + (uint32_t)i * 8u + (uint32_t)axis;
}
__host__ __device__ __forceinline__ uint32_t dim_final_gather(int i, int axis) {  // 0,1 BSDF 2D; 2 component
    return 0x600000u + (uint32_t)i * 4u + (uint32_t)axis;
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
    k.mode = W.sampler;
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

// traceDirect with highQuality false (direct_lighting.cpp:236-262): n lights chosen by power, one
// light and one BSDF sample each, from the branch key's streams
__device__ void direct_low_quality(const DScene& S, int n, const Bsdf& B, const HitContext& HC, float3 wi, float3 start,
                                   float lam, float T, uint32_t slot, uint32_t key, const SampleKey& skey,
                                   ShadowWriter& sw) {
    if (S.n_lights <= 0) return;
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
        estimate_light(S, B, HC, wi, start, l, 1, nb, lam, T / ((float)n * pc), slot, sw, u);
    }
}

template <bool TEX>
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
        HC = hit_context(S, o, d, (uint32_t)h.prim, h.t);
        // the camera vertex carries the camera's ray differentials (texture filtering); reflected
        // and transmitted tasks carry none
        if (TEX && gen == 0) camera_footprint(S, HC, (uint32_t)h.prim, W.cam, dkey(W, W.first_path + p), W.width, W.height);
        if (HC.mat < 0) {
            n_ch = more ? 1u : 0u;  // no shader: continue through the surface
        } else {
            M = S.mats[HC.mat];
            lam = P.lam[p];
            if (M.type != LIAR_MAT_NONE) {
                B = make_bsdf<TEX>(S, M, HC, lam);
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
    // a diffuse component do (estimateCaustics, estimateRadiance); high-quality ones gather their
    // indirect light with final gather rays instead of the radiance estimate (photon_mapper.cpp:490-507)
    const bool query = W.pm != 0 && shading && HC.mat >= 0 &&
                       (W.pm == 2 || (has_bsdf && has_caps(B.caps, CAP_DIFF)));
    const uint32_t n_fg = (query && W.pm == 1 && hq && W.fg_rays > 0) ? (uint32_t)W.fg_rays : 0u;
    if (W.pm != 0) {  // uniform over the launch: every lane of the warp takes the reservation
        const uint32_t qi = warp_reserve(W.q_count, query ? 1u : 0u);
        if (query) {
            W.q_pos[3 * (size_t)qi] = HC.target.x;
            W.q_pos[3 * (size_t)qi + 1] = HC.target.y;
            W.q_pos[3 * (size_t)qi + 2] = HC.target.z;
            W.q_task[qi] = q | (n_fg > 0 ? kNoRadiance : 0u);
        }
    }
    if (W.fg_rays > 0) {  // uniform as well
        const uint32_t gbase = warp_reserve(W.fg.count, n_fg);
        if (n_fg > 0) {
            // gatherIndirect (photon_mapper.cpp:1060-1146): BSDF samples of the reflective diffuse part
            const SampleKey skey = dkey(W, W.first_path + p);
            const float3 md = -d;
            float3 wi = mk(dot(md, HC.u), dot(md, HC.v), dot(md, HC.N));
            wi.z = fmaxf(wi.z, kEps);
            const float3 start = HC.target + (10.0f * kTol) * HC.N;
            for (uint32_t i = 0; i < n_fg; ++i) {
                const uint32_t gi = gbase + i;
                const BsdfSample bs = bsdf_sample(B, wi, sample_dim(skey, dim_final_gather((int)i, 0), true),
                                                  sample_dim(skey, dim_final_gather((int)i, 1), true),
                                                  sample_dim(skey, dim_final_gather((int)i, 2), true), CAP_REFL | CAP_DIFF);
                W.fg.slot[gi] = p;
                W.fg.meta[gi] = (uint32_t)(gen + 1);
                W.fg.key[gi] = child_key(key, 0x200u + i);
                if (bs.ok()) {
                    const float3 wd = bs.wo.x * HC.u + bs.wo.y * HC.v + bs.wo.z * HC.N;
                    put_ray(W.fg.rays, gi, start, wd, kTol, INFINITY);
                    W.fg.T[gi] = T * bs.value * (fabsf(bs.wo.z) / ((float)n_fg * bs.pdf));
                } else {
                    put_void_ray(W.fg.rays, gi);
                    W.fg.T[gi] = 0.0f;
                }
            }
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
                } else {
                    direct_low_quality(S, W.n_secondary, B, HC, wi, start, lam, T, p, key, skey, sw);
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
enum { kEstRadiance = 0, kEstCaustics = 1, kEstIrradiance = 2, kEstIrradianceMap = 3 };

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

// estimateRadiance from the nearest irradiance point j (photon_mapper.cpp:1290-1304): the BSDF
// from the viewer toward the point's normal times the point's irradiance at lam
__device__ float irradiance_map_radiance(const DScene& S, const PmIrradiance& I, const DRecovery& R,
                                         const HitContext& HC, float3 d, float lam, int32_t j) {
    if (j < 0 || (uint64_t)j >= I.n) return 0.0f;
    const liar_material Mat = S.mats[HC.mat];
    if (Mat.type == LIAR_MAT_NONE) return 0.0f;
    const Bsdf B = make_bsdf(S, Mat, HC, lam);
    if (!has_caps(B.caps, CAP_DIFF)) return 0.0f;
    const float3 md = -d;
    float3 wi = mk(dot(md, HC.u), dot(md, HC.v), dot(md, HC.N));
    wi.z = fmaxf(wi.z, kEps);
    const float3 n = mk(I.normal[3 * (size_t)j], I.normal[3 * (size_t)j + 1], I.normal[3 * (size_t)j + 2]);
    const BsdfOut be = bsdf_evaluate(B, wi, mk(dot(n, HC.u), dot(n, HC.v), dot(n, HC.N)), CAP_ALL);
    if (!(be.pdf > 0.0f) || be.value == 0.0f) return 0.0f;
    RecoveryBlend b;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        b.idx[c] = I.blend_idx[3 * (size_t)j + c];
        b.w[c] = I.blend_w[3 * (size_t)j + c];
    }
    return be.value * recovery_eval(R, b, lam, false);
}

// one thread per queried vertex: the vertex's BSDF against the k nearest photons of one map
//   kEstRadiance:   sum f(w, w_p) Phi_p(lam) / (pi r^2), f without its specular and glossy parts,
//                   at least two photons (estimateRadiance without an irradiance map)
//   kEstCaustics:   the same with the Gaussian filter w = alpha (1 - (1 - e^(-beta d^2 / 2r^2)) /
//                   (1 - e^-beta)), alpha 0.918, beta 1.953, f's diffuse part (estimateCaustics)
//   kEstIrradiance: the XYZ of the photons arriving from the normal's side over pi r^2, as a
//                   spectrum at lam (isVisualizingPhotonMap: estimateIrradianceImpl)
//   kEstIrradianceMap: f(w, n_i) E_i(lam) of the nearest irradiance point i within the radius
//                   (estimateRadiance with the precomputed irradiance map, :1290-1304)
// r^2 is the squared distance of the farthest photon found; the result, times the task's weight,
// is added to the sample's radiance
__global__ void __launch_bounds__(128) k_pm_estimate(DScene S, DParams W, DSamples P, DTasks tin,
                                                     const liar_hit* __restrict__ hits, const uint32_t* __restrict__ q_task,
                                                     uint32_t n_q, PmMap M, PmIrradiance I, DRecovery R, int kind,
                                                     const int32_t* __restrict__ g_idx, const float* __restrict__ g_d2,
                                                     const int32_t* __restrict__ g_cnt) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_q) return;
    if ((kind == kEstRadiance || kind == kEstIrradianceMap) && (q_task[i] & kNoRadiance)) return;
    const int k = kind == kEstIrradianceMap ? 1 : M.k;
    const int cnt = min(g_cnt[i], k);
    if (cnt < (kind == kEstIrradiance || kind == kEstIrradianceMap ? 1 : 2)) return;
    const uint32_t q = q_task[i] & ~kNoRadiance;
    const uint32_t p = tin.slot[q];
    const float T = tin.T[q];
    const float4 r0 = reinterpret_cast<const float4*>(tin.rays + q)[0];
    const float4 r1 = reinterpret_cast<const float4*>(tin.rays + q)[1];
    const float3 d = mk(r1.x, r1.y, r1.z);
    HitContext HC = hit_context(S, mk(r0.x, r0.y, r0.z), d, (uint32_t)hits[q].prim, hits[q].t);
    if (S.n_tex > 0 && (tin.meta[q] & 0xffu) == 0u)  // a camera vertex: its footprint, as k_dl_shade
        camera_footprint(S, HC, (uint32_t)hits[q].prim, W.cam, dkey(W, W.first_path + p), W.width, W.height);
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
    } else if (kind == kEstIrradianceMap) {
        result = irradiance_map_radiance(S, I, R, HC, d, lam, idx[0]);
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

// ---- final gathering (photon_mapper.cpp:1060-1251)

// the hits of the gather rays: a hit on an object without a shader continues through it
// (traceGatherRay's "entering or leaving something"); every other hit becomes a query of the map
// that answers estimateRadiance there (the irradiance map, else the global map)
__global__ void __launch_bounds__(128) k_fg_prep(DScene S, DTasks g, const liar_hit* __restrict__ hits, uint32_t n_g,
                                                 DTasks next, float* q_pos, uint32_t* q_task, uint32_t* q_count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n_g;
    bool cont = false, query = false;
    float3 point = mk(0, 0, 0);
    float4 r0 = make_float4(0, 0, 0, 0), r1 = make_float4(0, 0, 1, 0);
    liar_hit h{-1, 0.0f};
    if (valid && g.T[i] != 0.0f) {
        h = hits[i];
        if (h.prim >= 0) {
            r0 = reinterpret_cast<const float4*>(g.rays + i)[0];
            r1 = reinterpret_cast<const float4*>(g.rays + i)[1];
            const int mi = S.obj_mat[prim_object(S, (uint32_t)h.prim)];
            if (mi < 0) cont = true;
            else {
                query = true;
                point = mk(r0.x, r0.y, r0.z) + h.t * mk(r1.x, r1.y, r1.z);
            }
        }
    }
    const uint32_t qi = warp_reserve(q_count, query ? 1u : 0u);
    if (query) {
        q_pos[3 * (size_t)qi] = point.x;
        q_pos[3 * (size_t)qi + 1] = point.y;
        q_pos[3 * (size_t)qi + 2] = point.z;
        q_task[qi] = i;
    }
    const uint32_t ci = warp_reserve(next.count, cont ? 1u : 0u);
    if (cont) {
        put_ray(next.rays, ci, mk(r0.x, r0.y, r0.z), mk(r1.x, r1.y, r1.z), h.t + kTol, r1.w);
        next.slot[ci] = g.slot[i];
        next.T[ci] = g.T[i];
        next.meta[ci] = g.meta[i];
        next.key[ci] = g.key[i];
    }
}

// the radiance a gather ray brings back (traceGatherRay, photon_mapper.cpp:1150-1190): the map
// estimate at its hit, or, where the hit is closer than that estimate's radius at the first gather
// stage, numSecondaryGatherRays more gather rays and the low-quality direct light from there
// (gatherSecondary, :1195-1219)
__global__ void __launch_bounds__(128) k_fg_shade(DScene S, DParams W, DSamples P, DTasks g,
                                                  const liar_hit* __restrict__ hits, const uint32_t* __restrict__ q_task,
                                                  uint32_t n_q, PmMap M, PmIrradiance I, DRecovery R,
                                                  const int32_t* __restrict__ g_idx, const float* __restrict__ g_d2,
                                                  const int32_t* __restrict__ g_cnt, DTasks next, DShadows sh) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n_q;
    uint32_t gi = 0, p = 0, meta = 0, key = 0;
    float Tg = 0.0f, lam = 0.0f;
    float3 o = mk(0, 0, 0), d = mk(0, 0, 1);
    float t = 0.0f;
    HitContext HC;
    HC.mat = -1;
    HC.light = -1;
    Bsdf B{};
    bool bsdf_ok = false, secondary = false;
    float radiance = 0.0f;
    if (valid) {
        gi = q_task[i];
        p = g.slot[gi];
        Tg = g.T[gi];
        meta = g.meta[gi];
        key = g.key[gi];
        const float4 r0 = reinterpret_cast<const float4*>(g.rays + gi)[0];
        const float4 r1 = reinterpret_cast<const float4*>(g.rays + gi)[1];
        o = mk(r0.x, r0.y, r0.z);
        d = mk(r1.x, r1.y, r1.z);
        const liar_hit h = hits[gi];
        t = h.t;
        HC = hit_context(S, o, d, (uint32_t)h.prim, h.t);
        lam = P.lam[p];
        const liar_material Mat = S.mats[HC.mat];
        if (Mat.type != LIAR_MAT_NONE) {
            B = make_bsdf(S, Mat, HC, lam);
            bsdf_ok = true;
        }
        // estimateRadiance: nothing without a diffuse part (and its radius stays infinite)
        float sqr = INFINITY;
        if (bsdf_ok && has_caps(B.caps, CAP_DIFF)) {
            if (I.n > 0) {
                const int32_t j = g_cnt[i] > 0 ? g_idx[i] : -1;
                if (j < 0) {
                    sqr = M.radius;  // the reference assigns the radius, not its square (:1295)
                } else {
                    sqr = I.r2[j];
                    radiance = irradiance_map_radiance(S, I, R, HC, d, lam, j);
                }
            } else {
                const int k = M.k, cnt = min(g_cnt[i], k);
                if (cnt < 2) {
                    sqr = M.radius;  // as above (:1316)
                } else {
                    sqr = g_d2[(size_t)i * k + cnt - 1];
                    const float3 md = -d;
                    float3 wi = mk(dot(md, HC.u), dot(md, HC.v), dot(md, HC.N));
                    wi.z = fmaxf(wi.z, kEps);
                    for (int j = 0; j < cnt; ++j) {
                        const int32_t ph = g_idx[(size_t)i * k + j];
                        if (ph < 0 || (uint64_t)ph >= M.n) continue;
                        const float3 om = mk(M.omega_in[3 * (size_t)ph], M.omega_in[3 * (size_t)ph + 1],
                                             M.omega_in[3 * (size_t)ph + 2]);
                        const BsdfOut be = bsdf_evaluate(B, wi, mk(dot(om, HC.u), dot(om, HC.v), dot(om, HC.N)),
                                                         CAP_ALL & ~CAP_SPEC & ~CAP_GLOSSY);
                        if (!(be.pdf > 0.0f) || be.value == 0.0f) continue;
                        radiance += be.value * photon_power(M, R, ph, lam);
                    }
                    radiance /= 3.14159265358979323846f * sqr;
                }
            }
        }
        secondary = t * t < sqr && !(meta & kStage1) && W.fg_secondary > 0;
    }
    // gatherSecondary: the second stage's rays and shadow rays, reserved exactly
    const uint32_t n_ch = (secondary && bsdf_ok) ? (uint32_t)W.fg_secondary : 0u;
    const uint32_t n_sh = (secondary && bsdf_ok && S.n_lights > 0) ? 2u * (uint32_t)W.n_secondary : 0u;
    ShadowWriter sw{sh, warp_reserve(sh.count, n_sh), 0u, n_sh};
    const uint32_t cbase = warp_reserve(next.count, n_ch);
    if (valid && !secondary && radiance != 0.0f) atomicAdd(&P.L[p], Tg * radiance);
    if (n_ch > 0) {
        const SampleKey skey = dkey(W, W.first_path + p);
        const float3 md = -d;
        float3 wi = mk(dot(md, HC.u), dot(md, HC.v), dot(md, HC.N));
        wi.z = fmaxf(wi.z, kEps);
        const float3 target = o + t * d;
        for (uint32_t c = 0; c < n_ch; ++c) {
            const uint32_t ci = cbase + c;
            const uint32_t ck = child_key(key, 0x300u + c);
            const BsdfSample bs = bsdf_sample(B, wi, sample_dim(skey, dim_branch(ck, 0x2000u), false),
                                              sample_dim(skey, dim_branch(ck, 0x2001u), false),
                                              sample_dim(skey, dim_branch(ck, 0x2002u), false), CAP_REFL | CAP_DIFF);
            next.slot[ci] = p;
            next.meta[ci] = (meta & 0xffu) + 1u | kStage1;
            next.key[ci] = ck;
            if (bs.ok()) {
                put_ray(next.rays, ci, target, bs.wo.x * HC.u + bs.wo.y * HC.v + bs.wo.z * HC.N, kTol, INFINITY);
                next.T[ci] = Tg * bs.value * (fabsf(bs.wo.z) / ((float)n_ch * bs.pdf));
            } else {
                put_void_ray(next.rays, ci);
                next.T[ci] = 0.0f;
            }
        }
        direct_low_quality(S, W.n_secondary, B, HC, wi, HC.target + (10.0f * kTol) * HC.N, lam, Tg, p, key, skey, sw);
    }
    sw.finish(p);
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
    // final gathering: two queues of gather rays (48 B each, as tasks) and their hits
    void* fg[2] = {nullptr, nullptr};
    size_t n_fg[2] = {0, 0};
    liar_hit* fg_hits = nullptr;
    size_t fg_hits_cap = 0;
};

DirectBuffers* direct_buffers(liar_gpu_ctx* ctx) {
    for (auto& ext : ctx->extensions)
        if (ext.first == "direct") return static_cast<DirectBuffers*>(ext.second);
    DirectBuffers* b = new DirectBuffers();
    ctx->extensions.emplace_back("direct", b);
    ctx->on_destroy.push_back([b]() {
        for (void* p : {b->samples, b->tasks[0], b->tasks[1], b->shadows, (void*)b->hits, (void*)b->counters, b->queries,
                        b->gathers, b->fg[0], b->fg[1], (void*)b->fg_hits})
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

// the gather rays of one generation (n0 in queue 0): per stage trace them, let hits without a
// shader pass, query the map that estimates the radiance at the other hits, shade (estimate or
// second stage), then trace and add the shadow rays of the second stage; rays that pass and second
// stage rays form the next queue
int final_gather(liar_gpu_ctx* ctx, const liar_gpu_mesh* mesh, const DScene& S, DParams& W, const DSamples& P,
                 DirectBuffers* b, const PmMaps* pm, uint32_t n0, cudaStream_t st) {
    const PmMap& M = pm->map[kPmGlobal];
    const bool irr = pm->irr.n > 0;
    const int k = irr ? 1 : M.k;
    uint32_t n_g = n0;
    int cur = 0;
    for (int pass = 0; n_g > 0; ++pass) {
        if (pass > 32) return ctx_fail(ctx, LIAR_ERR_TIMEOUT, "final gather rays did not end after 32 passes");
        const uint64_t want_next = (uint64_t)n_g * (uint64_t)std::max(1, W.fg_secondary);
        const uint64_t want_sh = (uint64_t)n_g * 2ull * (uint64_t)W.n_secondary;
        if (want_next > (1ull << 31) || want_sh > (1ull << 31))
            return ctx_fail(ctx, LIAR_ERR_UNSUPPORTED, "final gather wave too large: set render.wave_paths lower");
        int rc = grow(ctx, &b->fg[cur ^ 1], &b->n_fg[cur ^ 1], want_next, 48, "final gather rays");
        if (!rc) rc = grow(ctx, &b->queries, &b->n_queries, n_g, 20, "final gather queries");
        if (!rc) rc = grow(ctx, &b->gathers, &b->n_gathers, (size_t)n_g * k, 8, "final gather neighbours");
        if (!rc) rc = grow(ctx, &b->shadows, &b->n_shadows, std::max<uint64_t>(want_sh, 1), 40, "final gather shadows");
        if (!rc && b->fg_hits_cap < std::max<uint64_t>(std::max<uint64_t>(want_sh, n_g), 1)) {
            void* hp = b->fg_hits;
            rc = grow(ctx, &hp, &b->fg_hits_cap, std::max<uint64_t>(want_sh, n_g), 8, "final gather hits");
            b->fg_hits = static_cast<liar_hit*>(hp);
        }
        if (rc) return rc;
        const DTasks g = task_view(b->fg[cur], b->n_fg[cur], b->counters + 4 + cur);
        const DTasks next = task_view(b->fg[cur ^ 1], b->n_fg[cur ^ 1], b->counters + 4 + (cur ^ 1));
        float* q_pos = static_cast<float*>(b->queries);
        uint32_t* q_task = reinterpret_cast<uint32_t*>(static_cast<char*>(b->queries) + b->n_queries * 12);
        int32_t* g_cnt = reinterpret_cast<int32_t*>(b->queries) + 4 * b->n_queries;
        int32_t* g_idx = static_cast<int32_t*>(b->gathers);
        float* g_d2 = reinterpret_cast<float*>(g_idx + b->n_gathers);
        DShadows sq;
        char* sc = static_cast<char*>(b->shadows);
        sq.rays = reinterpret_cast<liar_ray*>(sc);
        sq.slot = reinterpret_cast<uint32_t*>(sc + b->n_shadows * 32);
        sq.value = reinterpret_cast<float*>(sc + b->n_shadows * 36);
        sq.count = b->counters + 2;
        rc = trace_mesh_internal(ctx, mesh, g.rays, n_g, b->fg_hits, 0, st, kCounterWord + 10);
        if (rc) return rc;
        cudaError_t e = cudaMemsetAsync(b->counters + 4 + (cur ^ 1), 0, 4, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(b->counters + 2, 0, 8, st);  // shadows, queries
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "final gather counters");
        k_fg_prep<<<(n_g + 127) / 128, 128, 0, st>>>(S, g, b->fg_hits, n_g, next, q_pos, q_task, b->counters + 3);
        e = cudaMemcpyAsync(b->h_counters + 8, b->counters + 3, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "final gather queries");
        const uint32_t n_q = b->h_counters[8];
        if (n_q > 0) {
            rc = liar_gpu_photon_gather_device(ctx, irr ? pm->irr.grid : M.grid, q_pos, n_q, k, g_idx, g_d2, g_cnt, st);
            if (rc) return rc;
            k_fg_shade<<<(n_q + 127) / 128, 128, 0, st>>>(S, W, P, g, b->fg_hits, q_task, n_q, M, pm->irr, pm->rec, g_idx,
                                                          g_d2, g_cnt, next, sq);
            e = cudaGetLastError();
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "final gather shade launch");
        }
        e = cudaMemcpyAsync(b->h_counters + 8, b->counters, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "final gather queue sizes");
        const uint32_t n_sh = b->h_counters[8 + 2];
        const uint32_t n_next = b->h_counters[8 + 4 + (cur ^ 1)];
        if ((uint64_t)n_sh > want_sh || (uint64_t)n_next > want_next)
            return ctx_fail(ctx, LIAR_ERR_INVALID, "final gather queue overflow");
        if (n_sh > 0) {
            rc = trace_mesh_internal(ctx, mesh, sq.rays, n_sh, b->fg_hits, 1, st, kCounterWord + 10);
            if (rc) return rc;
            k_dl_shadow_add<<<(n_sh + 255) / 256, 256, 0, st>>>(sq, n_sh, b->fg_hits, P.L);
            e = cudaGetLastError();
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "final gather shadow launch");
        }
        cur ^= 1;
        n_g = n_next;
    }
    return LIAR_OK;
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
                                     : std::max<uint64_t>(4096, (1ull << 30) / (40ull * shadow_per_task + 64 +
                                                                                (pm ? 48ull * (uint64_t)pm->fg_rays : 0)));
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
    W.sampler = (uint32_t)R.sampler;
    W.seed = mix64(R.seed ^ mix64(0x51ed270b27ad0e0dull + (uint64_t)(uint32_t)R.first_sample));
    W.n_secondary = n_sec;
    W.glossy = R.trace_glossy < 0 ? 0u : CAP_GLOSSY;
    W.stats = stats;
    W.pm = pm ? (pm->visualize ? 2 : 1) : 0;
    W.pm_direct = pm ? pm->ray_direct : 1;
    W.q_pos = nullptr;
    W.q_task = nullptr;
    W.q_count = b->counters + 3;
    W.fg_rays = (pm && !pm->visualize) ? pm->fg_rays : 0;
    W.fg_secondary = pm ? pm->fg_secondary : 0;
    W.fg = DTasks{};
    W.fg.count = b->counters + 4;
    const DScene& S = scene_dscene(scene);
    const liar_gpu_mesh* mesh = scene_mesh(scene);
    for (uint64_t first = 0; first < total; first += wave) {
        if (ctx_cancel_requested(ctx)) return ctx_cancelled(ctx, st);
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
            if (ctx_cancel_requested(ctx)) return ctx_cancelled(ctx, st);
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
            if (!rc && W.fg_rays > 0) {
                rc = grow(ctx, &b->fg[0], &b->n_fg[0], (uint64_t)n_in * W.fg_rays, 48, "final gather rays");
                W.fg = task_view(b->fg[0], b->n_fg[0], b->counters + 4);
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
            if (e == cudaSuccess) e = cudaMemsetAsync(b->counters + 2, 0, 12, st);
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "reset queues");
            (S.n_tex > 0 ? k_dl_shade<true> : k_dl_shade<false>)<<<(n_in + 127) / 128, 128, 0, st>>>(S, W, P, tin, b->hits, n_in, tout, sq, (uint32_t)sh_hq);
            e = cudaGetLastError();
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "direct lighting shade launch");
            e = cudaMemcpyAsync(b->h_counters, b->counters, 5 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "direct lighting queue sizes");
            const uint32_t n_fg0 = W.fg_rays > 0 ? b->h_counters[4] : 0u;
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
                // the global estimate reads the irradiance map when there is one
                const bool irr = m == kPmGlobal && !pm->visualize && pm->irr.n > 0;
                const int k = irr ? 1 : M.k;
                rc = grow(ctx, &b->gathers, &b->n_gathers, (size_t)n_q * k, 8, "photon gathers");
                if (rc) return rc;
                int32_t* g_idx = static_cast<int32_t*>(b->gathers);
                float* g_d2 = reinterpret_cast<float*>(g_idx + b->n_gathers);
                int32_t* g_cnt = reinterpret_cast<int32_t*>(b->queries) + 4 * b->n_queries;  // after positions and tasks
                rc = liar_gpu_photon_gather_device(ctx, irr ? pm->irr.grid : M.grid, W.q_pos, n_q, k, g_idx, g_d2,
                                                   g_cnt, st);
                if (rc) return rc;
                const int kind = pm->visualize ? kEstIrradiance
                                               : (m == kPmGlobal ? (irr ? kEstIrradianceMap : kEstRadiance) : kEstCaustics);
                k_pm_estimate<<<(n_q + 127) / 128, 128, 0, st>>>(S, W, P, tin, b->hits, W.q_task, n_q, M, pm->irr,
                                                                  pm->rec, kind, g_idx, g_d2, g_cnt);
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
            if (n_fg0 > 0) {
                rc = final_gather(ctx, mesh, S, W, P, b, pm, n_fg0, st);
                if (rc) return rc;
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
