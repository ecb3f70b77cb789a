// render.cu -- wavefront spectral path tracer (the reference's AdjointPhotonTracer) on sm_100a.
//
// Replaces RenderEngine::render's per-sample loop (src/liar/kernel/render_engine.cpp:170-358)
// driving AdjointPhotonTracer::tracePhoton / shadeSurface / scatterSurface
// (src/liar/tracers/adjoint_photon_tracer.cpp:84-292). The recursion becomes a wavefront:
//
//   raygen   one thread per path: stratified screen / wavelength samples, camera ray
//            (PerspectiveCamera::doGenerateRay, cameras/perspective_camera.cpp:406-434),
//            Observer::sample for the wavelength (kernel/observer.cpp:283-317)
//   extend   the closest-hit trace kernel over the compacted ray queue
//   shade    one thread per queue entry: emission, BSDF set-up at the wavelength, one-sample MIS
//            between BSDF and light sampling, Russian roulette, then the next ray is appended
//            to the output queue (one atomicAdd per warp: ballot + popc compaction); finished
//            paths add their XYZ to the film
//
// The estimator is the reference's: there are no shadow rays; the light-sampling branch
// continues the path toward the light and the emission is picked up when that ray hits it.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <functional>
#include <new>
#include <vector>

#include "../../include/liar_gpu.h"
#include "ctx.h"
#include "photon_mapper.h"
#include "render_dev.cuh"

namespace liar_gpu {
const DRecovery* ctx_recovery(liar_gpu_ctx* ctx);  // recovery.cu
}

using namespace liar_gpu;
using namespace liar_gpu::rt;

struct liar_gpu_scene {
    int device = -1;
    uint64_t uid = 0;  // unique per upload in the process (keys caches of derived data)
    liar_gpu_mesh* mesh = nullptr;
    std::vector<void*> buffers;  // device allocations owned by the scene
    DScene d{};
    size_t n_triangles = 0;
    std::vector<liar_light> h_lights;        // host copies for launch planning
    std::vector<liar_material> h_materials;
};

namespace {

template <class T>
int upload(liar_gpu_ctx* ctx, liar_gpu_scene* s, const T* host, size_t n, const T** dev, const char* what) {
    *dev = nullptr;
    if (n == 0) return LIAR_OK;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, n * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return ctx_cuda(ctx, e, what);
    }
    s->buffers.push_back(p);
    e = cudaMemcpy(p, host, n * sizeof(T), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, what);
    *dev = static_cast<const T*>(p);
    return LIAR_OK;
}

// ---- path state (structure of arrays, one entry per path of the wave)
struct Paths {
    float* lam;        // wavelength (m)
    float* lam_pdf;    // its pdf
    float* T;          // throughput
    float* L;          // radiance gathered so far
    float* alpha;      // 1 once the camera ray hit something
    int32_t* gen;      // generation of the ray in flight
};

struct Queue {
    liar_ray* rays;
    uint32_t* path;
    uint32_t* count;   // device counter
};

struct WaveParams {
    liar_camera cam;
    int width, height, spp, max_gen, max_depth;
    uint32_t sampler;      // SAMPLER_* mode bits (sampler.h)
    uint64_t seed;
    uint64_t first_path;   // global index of the wave's first path
    FilmSpec film;
};

__device__ __forceinline__ SampleKey key_of(const WaveParams& W, uint64_t gpath) {
    SampleKey k;
    k.seed = W.seed;
    k.pixel = (uint32_t)(gpath / (uint64_t)W.spp);
    k.sample = (uint32_t)(gpath % (uint64_t)W.spp);
    k.spp = (uint32_t)W.spp;
    k.mode = W.sampler;
    return k;
}

// appends (ray, path) to q with one atomic per warp
__device__ __forceinline__ void queue_push(const Queue& q, bool want, const liar_ray& r, uint32_t path) {
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

__device__ void splat(const DScene& S, const WaveParams& W, uint64_t gpath, float lam, float lam_pdf, float L,
                      float alpha) {
    float3 xyz = mk(0, 0, 0);
    if (lam_pdf > 0.0f) {
        // Spectral::xyz in Single mode: v / pdf * sensitivity(lambda) (kernel/spectral.cpp:212-220)
        const float s = L / lam_pdf;
        const float3 c = observer_sensitivity(S, lam);
        xyz = mk(s * c.x, s * c.y, s * c.z);
    }
    film_splat(W.film, key_of(W, gpath), xyz, alpha);
}

__global__ void __launch_bounds__(256) k_raygen(DScene S, WaveParams W, Paths P, Queue out, uint32_t n_paths,
                                                unsigned long long* stats) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool want = false;
    liar_ray r{};
    if (i < n_paths) {
        const uint64_t g = W.first_path + i;
        const SampleKey k = key_of(W, g);
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
    queue_push(out, want, r, i);
}

// the whole of tracePhoton after the intersection, for one queue entry
template <bool TEX>
__global__ void __launch_bounds__(128) k_shade(DScene S, WaveParams W, Paths P, Queue in, const liar_hit* hits,
                                               uint32_t n_in, const uint32_t* __restrict__ n_dev, Queue out,
                                               unsigned long long* stats) {
    // n_dev: the queue's size in device memory when the host launched with an upper bound
    if (n_dev) n_in = min(n_in, *n_dev);
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    bool want = false;
    liar_ray nr{};
    uint32_t p = 0;
    uint32_t n_hit = 0;
    if (q < n_in) {
        p = in.path[q];
        const float4 r0 = reinterpret_cast<const float4*>(in.rays + q)[0];
        const float4 r1 = reinterpret_cast<const float4*>(in.rays + q)[1];
        const float3 o = mk(r0.x, r0.y, r0.z), d = mk(r1.x, r1.y, r1.z);
        const liar_hit h = hits[q];
        const uint64_t g = W.first_path + p;
        const SampleKey key = key_of(W, g);
        const int gen = P.gen[p];
        float T = P.T[p], L = P.L[p];
        const float lam = P.lam[p];
        bool alive = false;
        float3 next_o = mk(0, 0, 0), next_d = mk(0, 0, 1);
        float next_tmin = kTol, next_tmax = INFINITY;

        if (h.prim < 0) {
            // the sky is an object at a fixed distance (LightSky::doIntersect)
            if (S.sky_light >= 0 && S.sky_distance > r0.w * (1.0f + kTol) && S.sky_distance < r1.w * (1.0f - kTol)) {
                if (gen == 0) P.alpha[p] = 1.0f;
                if (gen > 0) L += T * spec_eval(S, S.lights[S.sky_light].spectrum, lam, false);
                // no shader: the ray continues past the sky and finds nothing
            }
        } else {
            ++n_hit;
            if (gen == 0) P.alpha[p] = 1.0f;
            // ---- IntersectionContext of the hit (re-intersection, normals flipped toward -d, frame)
            HitContext H = hit_context(S, o, d, (uint32_t)h.prim, h.t);
            // the camera vertex carries the camera's ray differentials (texture filtering)
            if (TEX && gen == 0) camera_footprint(S, H, (uint32_t)h.prim, W.cam, key, W.width, W.height);
            const int light = H.light;
            const int mi = H.mat;
            const float3 target = H.target, ng = H.ng, N = H.N, u = H.u, v = H.v;
            if (gen > 0 && light >= 0) {
                // LightArea::doEmission: radiance of the light object that was hit
                L += T * spec_eval(S, S.lights[light].spectrum, lam, false);
            }
            // the shader's emission counts unless a light was hit past the camera vertex (the
            // reference asks the object for its light only at generations > 0)
            const bool shader_emits = gen == 0 || light < 0;
            if (mi < 0) {
                // no shader: entering or leaving something, continue through (bound(ray, t + tolerance, far))
                alive = true;
                next_o = o;
                next_d = d;
                next_tmin = h.t + kTol;
                next_tmax = r1.w;
            } else if (S.mats[mi].type == LIAR_MAT_NONE) {
                // a shader without a BSDF (Unshaded): its emission, and the path ends
                if (shader_emits && S.mats[mi].emission >= 0) L += T * spec_eval(S, S.mats[mi].emission, lam, false);
            } else {
                const liar_material M = S.mats[mi];
                if (shader_emits && M.emission >= 0) L += T * spec_eval(S, M.emission, lam, false);
                const Bsdf B = make_bsdf<TEX>(S, M, H, lam);  // Shader::bsdf at this wavelength
                const float3 md = -d;
                float3 wi = mk(dot(md, u), dot(md, v), dot(md, N));
                wi.z = fmaxf(wi.z, kEps);
                // ---- scatterSurface: one-sample MIS (adjoint_photon_tracer.cpp:212-292)
                const bool strat = gen < W.max_gen;
                const uint32_t base = DIM_GEN0 + DIMS_PER_GEN * (uint32_t)gen;
                const float strategy_pdf = (has_caps(B.caps, CAP_DIFF) || has_caps(B.caps, CAP_GLOSSY)) ? 0.5f : 1.0f;
                BsdfSample out{mk(0, 0, 0), 0.0f, 0.0f};
                bool ok = false;
                // the strategy's own direction (divergent: BSDF sample or light sample), then the
                // other lights' emission densities along it in one loop every lane runs together,
                // then the strategy's weight (the sums keep the light order of both branches)
                const bool by_bsdf = sample_dim(key, base + OFF_STRATEGY, strat) < strategy_pdf;
                bool have = false;
                int k = -1;
                float3 dir = mk(0, 0, 1);
                float acc = 0.0f;
                if (by_bsdf) {
                    out = bsdf_sample(B, wi, sample_dim(key, base + OFF_BSDF, strat), sample_dim(key, base + OFF_BSDF + 1, strat),
                                      sample_dim(key, base + OFF_COMPONENT, strat), CAP_ALL);
                    if (out.ok()) {
                        out.pdf *= strategy_pdf;
                        dir = out.wo.x * u + out.wo.y * v + out.wo.z * N;
                        have = true;
                    }
                } else if (S.n_lights > 0) {
                    const float uc = sample_dim(key, base + OFF_LIGHT_CHOICE, strat);
                    k = lower_bound_f(S.light_cdf, S.n_lights, uc);
                    if (k > S.n_lights - 1) k = S.n_lights - 1;
                    const float pc = light_choice_pdf(S, k);
                    if (pc > 0.0f) {
                        const LightSample ls = light_sample(S, k, target, sample_dim(key, base + OFF_LIGHT, strat),
                                                            sample_dim(key, base + OFF_LIGHT + 1, strat), lam);
                        if (ls.pdf > 0.0f) {
                            acc = pc * ls.pdf;
                            dir = ls.dir;
                            have = true;
                        }
                    }
                }
                if (have) {
                    for (int l = 0; l < S.n_lights; ++l) {
                        if (l == k) continue;
                        const LightEmission e = light_emission(S, l, target, dir, lam);
                        if (e.pdf > 0.0f) acc += light_choice_pdf(S, l) * e.pdf;
                    }
                    acc *= (1.0f - strategy_pdf);
                    if (by_bsdf) {
                        out.value *= power_heuristic(out.pdf, acc);
                        ok = out.ok();
                    } else {
                        const float3 wo = mk(dot(dir, u), dot(dir, v), dot(dir, N));
                        const BsdfOut be = bsdf_evaluate(B, wi, wo, CAP_ALL);
                        if (be.pdf > 0.0f && be.value != 0.0f) {
                            out.wo = wo;
                            out.value = be.value * power_heuristic(acc, be.pdf * strategy_pdf);
                            out.pdf = acc;
                            ok = out.ok();
                        }
                    }
                }
                if (ok) {
                    // shadeSurface continues along the scattered direction (adjoint_photon_tracer.cpp:170-186)
                    const float cos_t = out.wo.z;
                    next_o = target + ((cos_t > 0.0f ? 10.0f : -10.0f) * kTol) * ng;
                    next_d = out.wo.x * u + out.wo.y * v + out.wo.z * N;
                    next_tmin = kTol;
                    next_tmax = INFINITY;
                    T *= out.value * (fabsf(cos_t) / out.pdf);
                    alive = true;
                }
            }
        }
        if (alive) {
            const int ng1 = gen + 1;
            if (W.max_depth > 0 && ng1 >= W.max_depth) {
                alive = false;
            } else if (ng1 >= W.max_gen) {
                // Russian roulette at the start of tracePhoton (adjoint_photon_tracer.cpp:86-100)
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
            splat(S, W, g, lam, P.lam_pdf[p], L, P.alpha[p]);
        }
    }
    queue_push(out, want, nr, p);
    // statistics: segments traced and hits
    const uint32_t lane = threadIdx.x & 31u;
    unsigned long long segs = (q < n_in) ? 1ull : 0ull, hh = n_hit;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        segs += __shfl_down_sync(0xffffffffu, segs, o);
        hh += __shfl_down_sync(0xffffffffu, hh, o);
    }
    if (lane == 0 && segs) {
        atomicAdd(stats + 1, segs);
        atomicAdd(stats + 2, hh);
    }
}

}  // namespace

// ------------------------------------------------------------------------------------------------

namespace {

struct RenderBuffers {
    size_t cap = 0;
    void* mem = nullptr;
    Paths P{};
    Queue q[2]{};
    liar_hit* hits = nullptr;
    unsigned long long* stats = nullptr;  // [0] paths [1] segments [2] hits
    uint32_t* h_count = nullptr;          // pinned, two slots
    cudaEvent_t ev[2] = {nullptr, nullptr};  // the copies into them
};

RenderBuffers* render_buffers(liar_gpu_ctx* ctx) {
    static_assert(sizeof(liar_ray) == 32, "ray layout");
    for (auto& ext : ctx->extensions)
        if (ext.first == "render") return static_cast<RenderBuffers*>(ext.second);
    RenderBuffers* rb = new RenderBuffers();
    ctx->extensions.emplace_back("render", rb);
    ctx->on_destroy.push_back([rb]() {
        if (rb->mem) cudaFree(rb->mem);
        if (rb->stats) cudaFree(rb->stats);
        if (rb->h_count) cudaFreeHost(rb->h_count);
        for (cudaEvent_t e : rb->ev)
            if (e) cudaEventDestroy(e);
        delete rb;
    });
    return rb;
}

int ensure_render_buffers(liar_gpu_ctx* ctx, RenderBuffers* rb, size_t n) {
    if (!rb->stats) {
        cudaError_t e = cudaMalloc((void**)&rb->stats, 4 * sizeof(unsigned long long));
        if (e == cudaSuccess) e = cudaMallocHost((void**)&rb->h_count, 2 * sizeof(uint32_t));
        for (int k = 0; k < 2 && e == cudaSuccess; ++k)
            if (!rb->ev[k]) e = cudaEventCreateWithFlags(&rb->ev[k], cudaEventDisableTiming);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "render statistics buffers");
    }
    if (rb->cap >= n) return LIAR_OK;
    if (rb->mem) cudaFree(rb->mem);
    rb->mem = nullptr;
    rb->cap = 0;
    // per path: 6 state words; per queue slot (x2): 32 B ray + 4 B path; hits 8 B; 2 counters;
    // plus the 256-byte rounding of each of the 13 pieces
    const size_t bytes = n * (6 * 4 + 2 * (32 + 4) + 8) + 13 * 256;
    cudaError_t e = cudaMalloc(&rb->mem, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return ctx_cuda(ctx, e, "render wave buffers");
    }
    char* p = static_cast<char*>(rb->mem);
    auto take = [&](size_t b) {
        char* r = p;
        p += (b + 255) & ~size_t(255);
        return r;
    };
    rb->q[0].rays = reinterpret_cast<liar_ray*>(take(n * 32));
    rb->q[1].rays = reinterpret_cast<liar_ray*>(take(n * 32));
    rb->hits = reinterpret_cast<liar_hit*>(take(n * 8));
    rb->q[0].path = reinterpret_cast<uint32_t*>(take(n * 4));
    rb->q[1].path = reinterpret_cast<uint32_t*>(take(n * 4));
    rb->P.lam = reinterpret_cast<float*>(take(n * 4));
    rb->P.lam_pdf = reinterpret_cast<float*>(take(n * 4));
    rb->P.T = reinterpret_cast<float*>(take(n * 4));
    rb->P.L = reinterpret_cast<float*>(take(n * 4));
    rb->P.alpha = reinterpret_cast<float*>(take(n * 4));
    rb->P.gen = reinterpret_cast<int32_t*>(take(n * 4));
    rb->q[0].count = reinterpret_cast<uint32_t*>(take(4));
    rb->q[1].count = reinterpret_cast<uint32_t*>(take(4));
    rb->cap = n;
    return LIAR_OK;
}

}  // namespace

extern "C" int liar_gpu_scene_upload(liar_gpu_ctx* ctx, const liar_scene_desc* desc, liar_gpu_scene** out) {
    if (!ctx || !desc || !out) return LIAR_ERR_INVALID;
    *out = nullptr;
    const liar_scene_desc& D = *desc;
    if (D.n_triangles == 0 && D.n_spheres == 0) return ctx_fail(ctx, LIAR_ERR_INVALID, "scene has no triangles");
    if (D.n_triangles > 0 && (!D.vertices || !D.triangles || !D.triangle_object))
        return ctx_fail(ctx, LIAR_ERR_INVALID, "scene has no triangles");
    if (D.n_spheres > 0 && (!D.spheres || !D.sphere_object)) return ctx_fail(ctx, LIAR_ERR_INVALID, "spheres missing");
    for (size_t k = 0; k < D.n_spheres; ++k) {
        const int32_t o = D.sphere_object[k];
        if (o < 0 || (size_t)o >= D.n_objects) return ctx_fail(ctx, LIAR_ERR_INVALID, "sphere %zu: object index out of range", k);
        const float* sp = D.spheres + 4 * k;
        if (!std::isfinite(sp[0]) || !std::isfinite(sp[1]) || !std::isfinite(sp[2]) || !(sp[3] > 0.0f) || !std::isfinite(sp[3]))
            return ctx_fail(ctx, LIAR_ERR_INVALID, "sphere %zu: centre not finite or radius not positive", k);
    }
    if (!D.object_material || !D.object_light || D.n_objects == 0) return ctx_fail(ctx, LIAR_ERR_INVALID, "scene has no objects");
    if (!D.observer || D.n_observer < 2) return ctx_fail(ctx, LIAR_ERR_INVALID, "observer table needs two or more rows");
    if (D.n_lights > 4096) return ctx_fail(ctx, LIAR_ERR_INVALID, "too many lights (limit 4096)");
    // validation of every index the kernels follow
    for (size_t k = 0; k < D.n_triangles; ++k) {
        const int32_t o = D.triangle_object[k];
        if (o < 0 || (size_t)o >= D.n_objects) return ctx_fail(ctx, LIAR_ERR_INVALID, "triangle %zu: object index out of range", k);
        if (D.triangle_normals)
            for (int c = 0; c < 3; ++c) {
                const int32_t ni = D.triangle_normals[3 * k + c];
                if (ni >= 0 && (size_t)ni >= D.n_normals)
                    return ctx_fail(ctx, LIAR_ERR_INVALID, "triangle %zu: normal index out of range", k);
            }
    }
    for (size_t k = 0; k < D.n_objects; ++k) {
        const int32_t m = D.object_material[k], l = D.object_light[k];
        if (m >= 0 && (size_t)m >= D.n_materials) return ctx_fail(ctx, LIAR_ERR_INVALID, "object %zu: material out of range", k);
        if (l >= 0 && (size_t)l >= D.n_lights) return ctx_fail(ctx, LIAR_ERR_INVALID, "object %zu: light out of range", k);
    }
    auto spec_ok = [&](int32_t s) { return s >= -1 && s < (int32_t)D.n_spectra; };
    for (size_t k = 0; k < D.n_materials; ++k) {
        const liar_material& m = D.materials[k];
        if (m.type < LIAR_MAT_NONE || m.type > LIAR_MAT_MIRROR) return ctx_fail(ctx, LIAR_ERR_INVALID, "material %zu: bad type", k);
        for (int c = 0; c < 4; ++c)
            if (!spec_ok(m.spec[c])) return ctx_fail(ctx, LIAR_ERR_INVALID, "material %zu: spectrum out of range", k);
        if (!spec_ok(m.emission)) return ctx_fail(ctx, LIAR_ERR_INVALID, "material %zu: emission out of range", k);
        for (int c = 0; c < 4; ++c)
            if (m.tex[c] < -1 || (m.tex[c] >= 0 && (size_t)m.tex[c] >= D.n_textures))
                return ctx_fail(ctx, LIAR_ERR_INVALID, "material %zu: texture out of range", k);
    }
    if (D.n_textures > 0 && !D.textures) return ctx_fail(ctx, LIAR_ERR_INVALID, "textures missing");
    if (D.n_textures > (1u << 20)) return ctx_fail(ctx, LIAR_ERR_INVALID, "too many textures (limit 2^20)");
    // every texture node must end at constants within 32 nodes (the lookup's bound), without cycles
    std::vector<int> tex_depth(D.n_textures, 0);  // 0: not visited, -1: being visited, else its depth
    std::vector<int> tex_post(D.n_textures, 0);   // the most ABS / AFFINE nodes on a path down from it
    const char* tex_err = nullptr;
    int tex_bad = -1;
    bool has_images = false, has_noise = false;
    std::function<int(int, int)> depth_of = [&](int t, int level) -> int {
        if (t < 0 || (size_t)t >= D.n_textures) return tex_err = "child out of range", -1;
        if (tex_depth[t] > 0) return tex_depth[t];
        if (tex_depth[t] < 0) return tex_err = "cycle", tex_bad = t, -1;
        if (level > 32) return tex_err = "more than 32 nested textures", tex_bad = t, -1;
        const liar_texture& T = D.textures[t];
        int d = 0;
        if (T.type == LIAR_TEX_CONSTANT) {
            if (T.spectrum < 0 || T.spectrum >= (int32_t)D.n_spectra) return tex_err = "spectrum out of range", tex_bad = t, -1;
            d = 1;
        } else if (T.type == LIAR_TEX_IMAGE) {
            // the mip table at `pixels` (see include/liar_gpu.h): level counts and mode, then per level
            // the offset of its pixels (from `pixels`) and its size, every level inside the pool
            const uint64_t np = D.n_texture_pixels;
            if (T.a <= 0 || T.b <= 0 || T.pixels < 0 || !D.texture_pixels || (uint64_t)T.pixels >= np)
                return tex_err = "image pixels out of range", tex_bad = t, -1;
            const float* hp = D.texture_pixels + 4 * (size_t)T.pixels;
            int32_t hdr[4];
            std::memcpy(hdr, hp, sizeof(hdr));
            const int n_u = hdr[0], n_v = hdr[1], mip = hdr[2];
            if (n_u < 1 || n_u > 32 || n_v < 1 || n_v > 32 || mip < 0 || mip > 2 || (mip != 2 && n_v != 1) ||
                (mip == 0 && n_u != 1) || (uint64_t)T.pixels + 1 + (uint64_t)n_u * n_v > np)
                return tex_err = "bad image mip table", tex_bad = t, -1;
            for (int lv = 0; lv < n_u * n_v; ++lv) {
                int32_t e[4];
                std::memcpy(e, hp + 4 * (1 + lv), sizeof(e));
                const uint64_t off = ((uint64_t)(uint32_t)e[1] << 31) | (uint64_t)(uint32_t)e[0];
                if (e[2] <= 0 || e[3] <= 0 || off < 1 + (uint64_t)n_u * n_v ||
                    (uint64_t)T.pixels + off + (uint64_t)e[2] * (uint64_t)e[3] > np)
                    return tex_err = "image mip level out of range", tex_bad = t, -1;
            }
            if (!(T.p[0] == 0.0f || T.p[0] == 1.0f || T.p[0] == 2.0f))
                return tex_err = "image anti-aliasing must be 0, 1 or 2", tex_bad = t, -1;
            has_images = true;
            d = 1;
        } else if (T.type == LIAR_TEX_NOISE) {
            if (T.pixels < 0 || !D.noise_tables || (uint64_t)T.pixels + 771 > (uint64_t)D.n_noise_tables)
                return tex_err = "noise tables out of range", tex_bad = t, -1;
            if (!(T.p[0] >= 0.0f && T.p[0] <= 64.0f && T.p[0] == std::floor(T.p[0])) || !std::isfinite(T.p[1]))
                return tex_err = "noise octaves must be an integer in 0..64 with a finite falloff", tex_bad = t, -1;
            has_noise = true;
            d = 1;
        } else if (T.type == LIAR_TEX_ABS || T.type == LIAR_TEX_AFFINE) {
            if (!std::isfinite(T.p[0]) || !std::isfinite(T.p[1])) return tex_err = "non-finite parameters", tex_bad = t, -1;
            tex_depth[t] = -1;
            const int da = depth_of(T.a, level + 1);
            if (da < 0) return -1;
            if (tex_post[T.a] + 1 > 8)
                return tex_err = "more than 8 Abs, Product, Sum or anti-aliased CheckerBoard nodes on a path", tex_bad = t, -1;
            tex_post[t] = tex_post[T.a] + 1;
            d = da + 1;
        } else if (T.type == LIAR_TEX_CHECKER || T.type == LIAR_TEX_GRID || T.type == LIAR_TEX_UV_TRANSFORM) {
            tex_depth[t] = -1;
            const int da = depth_of(T.a, level + 1);
            if (da < 0) return -1;
            int db = 0;
            if (T.type != LIAR_TEX_UV_TRANSFORM && (db = depth_of(T.b, level + 1)) < 0) return -1;
            d = std::max(da, db) + 1;
            // an anti-aliased CheckerBoard waits for both children: one more pending operator
            const int own = (T.type == LIAR_TEX_CHECKER && T.p[2] != 0.0f) ? 1 : 0;
            tex_post[t] = std::max(tex_post[T.a], T.type != LIAR_TEX_UV_TRANSFORM ? tex_post[T.b] : 0) + own;
            if (tex_post[t] > 8)
                return tex_err = "more than 8 Abs, Product, Sum or anti-aliased CheckerBoard nodes on a path", tex_bad = t, -1;
        } else {
            return tex_err = "bad type", tex_bad = t, -1;
        }
        if (d > 32) return tex_err = "more than 32 nested textures", tex_bad = t, -1;
        return tex_depth[t] = d;
    };
    for (size_t k = 0; k < D.n_textures; ++k)
        if (depth_of((int)k, 1) < 0) return ctx_fail(ctx, LIAR_ERR_INVALID, "texture %d: %s", tex_bad < 0 ? (int)k : tex_bad, tex_err);
    const DRecovery* rec = has_images ? ctx_recovery(ctx) : nullptr;
    if (has_images && !rec)
        return ctx_fail(ctx, LIAR_ERR_INVALID, "image textures need the context's recovery table (liar_gpu_set_recovery)");
    std::vector<float> spec_max(D.n_spectra, 0.0f);
    for (size_t k = 0; k < D.n_spectra; ++k) {
        const liar_spectrum& s = D.spectra[k];
        if (s.type == LIAR_SPEC_SAMPLED) {
            if (s.count < 2 || s.offset < 0 || (size_t)s.offset + 2 * (size_t)s.count > D.pool_size)
                return ctx_fail(ctx, LIAR_ERR_INVALID, "spectrum %zu: sampled table out of range", k);
            float mx = -INFINITY;
            for (int i = 0; i < s.count; ++i) mx = std::max(mx, D.spectrum_pool[s.offset + s.count + i]);
            spec_max[k] = s.p[0] > 0.0f ? s.p[0] : mx;  // p[0] > 0: the reflectance bound of a recovered colour
        } else if (s.type < 0 || s.type > LIAR_SPEC_CAUCHY) {
            return ctx_fail(ctx, LIAR_ERR_INVALID, "spectrum %zu: bad type", k);
        }
    }
    int sky = -1;
    std::vector<float> cdf(D.n_lights), area(D.n_lights, 0.0f), tri_cdf(D.n_triangles, 0.0f);
    double total = 0.0;
    for (size_t k = 0; k < D.n_lights; ++k) {
        const liar_light& L = D.lights[k];
        if (!spec_ok(L.spectrum) || L.spectrum < 0) return ctx_fail(ctx, LIAR_ERR_INVALID, "light %zu: spectrum out of range", k);
        if (L.type == LIAR_LIGHT_SKY) {
            if (sky >= 0) return ctx_fail(ctx, LIAR_ERR_UNSUPPORTED, "more than one sky light");
            sky = (int)k;
        } else if (L.type == LIAR_LIGHT_AREA_PARALLELOGRAM) {
            const double ux = L.u[0], uy = L.u[1], uz = L.u[2], vx = L.v[0], vy = L.v[1], vz = L.v[2];
            const double cx = uy * vz - uz * vy, cy = uz * vx - ux * vz, cz = ux * vy - uy * vx;
            area[k] = (float)std::sqrt(cx * cx + cy * cy + cz * cz);
        } else if (L.type == LIAR_LIGHT_AREA_MESH) {
            if (L.first_tri < 0 || L.n_tris <= 0 || (size_t)L.first_tri + (size_t)L.n_tris > D.n_triangles)
                return ctx_fail(ctx, LIAR_ERR_INVALID, "light %zu: triangle range out of range", k);
            if (L.n_tris > 1024) return ctx_fail(ctx, LIAR_ERR_UNSUPPORTED, "light %zu: mesh lights hold at most 1024 triangles", k);
            double acc = 0.0;
            std::vector<double> ar(L.n_tris);
            for (int i = 0; i < L.n_tris; ++i) {
                const uint32_t* t = D.triangles + 3 * (size_t)(L.first_tri + i);
                const float* a = D.vertices + 3 * t[0];
                const float* b = D.vertices + 3 * t[1];
                const float* c = D.vertices + 3 * t[2];
                const double e1[3] = {(double)b[0] - a[0], (double)b[1] - a[1], (double)b[2] - a[2]};
                const double e2[3] = {(double)c[0] - a[0], (double)c[1] - a[1], (double)c[2] - a[2]};
                const double nx = e1[1] * e2[2] - e1[2] * e2[1], ny = e1[2] * e2[0] - e1[0] * e2[2],
                             nz = e1[0] * e2[1] - e1[1] * e2[0];
                ar[i] = 0.5 * std::sqrt(nx * nx + ny * ny + nz * nz);
                acc += ar[i];
            }
            double run = 0.0;
            for (int i = 0; i < L.n_tris; ++i) {
                run += ar[i];
                tri_cdf[L.first_tri + i] = (float)(run / acc);
            }
            area[k] = (float)acc;
        } else if (L.type != LIAR_LIGHT_POINT) {
            return ctx_fail(ctx, LIAR_ERR_INVALID, "light %zu: bad type", k);
        }
        total += std::max(0.0f, L.power);
        cdf[k] = (float)total;
    }
    for (size_t k = 0; k < D.n_lights; ++k) cdf[k] = total > 0 ? (float)(cdf[k] / total) : (float)(k + 1) / D.n_lights;
    // observer: normalise so that the Y of the unit spectrum is 1 and build the sampling CDF
    // (Observer::Observer, kernel/observer.cpp:57-129)
    const size_t no = D.n_observer;
    std::vector<float> ow(no), oxyz(3 * no), odxyz(3 * no, 0.0f), ocdf(no);
    {
        std::vector<double> dX(3 * no);
        double prev = D.observer[0];
        ocdf[0] = 0.0f;
        double acc = 0.0;
        std::vector<double> cd(no, 0.0);
        for (size_t k = 0; k + 1 < no; ++k) {
            const double w = D.observer[4 * k], wn = D.observer[4 * (k + 1)];
            if (!(wn > w)) return ctx_fail(ctx, LIAR_ERR_INVALID, "observer wavelengths must increase");
            for (int c = 0; c < 3; ++c) {
                odxyz[3 * k + c] = (float)((D.observer[4 * (k + 1) + 1 + c] - D.observer[4 * k + 1 + c]) / (wn - w));
                dX[3 * k + c] = D.observer[4 * k + 1 + c] * ((wn - prev) / 2);
            }
            prev = w;
            acc += (std::fabs(D.observer[4 * k + 1]) + std::fabs(D.observer[4 * k + 2]) + std::fabs(D.observer[4 * k + 3]) +
                    std::fabs(D.observer[4 * (k + 1) + 1]) + std::fabs(D.observer[4 * (k + 1) + 2]) +
                    std::fabs(D.observer[4 * (k + 1) + 3])) * (wn - w);
            cd[k + 1] = acc;
        }
        const double wl = D.observer[4 * (no - 1)];
        for (int c = 0; c < 3; ++c) dX[3 * (no - 1) + c] = D.observer[4 * (no - 1) + 1 + c] * ((wl - prev) / 2);
        double Y = 0.0;
        for (size_t k = 0; k < no; ++k) Y += dX[3 * k + 1];
        if (!(Y > 0)) return ctx_fail(ctx, LIAR_ERR_INVALID, "observer has no luminance");
        for (size_t k = 0; k < no; ++k) {
            ow[k] = D.observer[4 * k];
            for (int c = 0; c < 3; ++c) {
                oxyz[3 * k + c] = (float)(D.observer[4 * k + 1 + c] / Y);
                odxyz[3 * k + c] = (float)(odxyz[3 * k + c] / Y);
            }
            ocdf[k] = (float)(cd[k] / acc);
        }
        ocdf[no - 1] = 1.0f;
    }

    int rc = ctx_activate(ctx);
    if (rc) return rc;
    liar_gpu_scene* s = new (std::nothrow) liar_gpu_scene();
    if (!s) return ctx_fail(ctx, LIAR_ERR_OOM, "host allocation");
    s->device = ctx->device;
    static std::atomic<uint64_t> next_uid{1};
    s->uid = next_uid.fetch_add(1);
    rc = mesh_build_with_spheres(ctx, D.vertices, D.n_vertices, D.triangles, D.n_triangles, D.spheres, D.n_spheres,
                                 nullptr, &s->mesh);
    DScene& d = s->d;
    if (!rc) rc = upload(ctx, s, D.vertices, 3 * D.n_vertices, &d.verts, "scene vertices");
    if (!rc) rc = upload(ctx, s, D.triangles, 3 * D.n_triangles, &d.tri_idx, "scene triangles");
    if (!rc) rc = upload(ctx, s, D.triangle_object, D.n_triangles, &d.tri_obj, "triangle objects");
    if (!rc && D.n_spheres) {
        const float* sp = nullptr;
        rc = upload(ctx, s, D.spheres, 4 * D.n_spheres, &sp, "spheres");
        d.spheres = reinterpret_cast<const float4*>(sp);
        if (!rc) rc = upload(ctx, s, D.sphere_object, D.n_spheres, &d.sphere_obj, "sphere objects");
    }
    d.n_tris = (uint32_t)D.n_triangles;
    if (!rc && D.normals && D.triangle_normals) {
        rc = upload(ctx, s, D.normals, 3 * D.n_normals, &d.normals, "normals");
        if (!rc) rc = upload(ctx, s, D.triangle_normals, 3 * D.n_triangles, &d.tri_nrm, "triangle normals");
    }
    if (!rc && D.triangle_uvs) rc = upload(ctx, s, D.triangle_uvs, 6 * D.n_triangles, &d.tri_uv, "triangle uvs");
    if (!rc) rc = upload(ctx, s, D.textures, D.n_textures, &d.texs, "textures");
    if (!rc && has_images) {
        const float* px = nullptr;
        rc = upload(ctx, s, D.texture_pixels, 4 * D.n_texture_pixels, &px, "texture pixels");
        d.tex_pixels = reinterpret_cast<const float4*>(px);
        d.rec = *rec;
    }
    if (!rc && has_noise) rc = upload(ctx, s, D.noise_tables, D.n_noise_tables, &d.noise_tables, "noise tables");
    if (!rc) rc = upload(ctx, s, D.object_material, D.n_objects, &d.obj_mat, "object materials");
    if (!rc) rc = upload(ctx, s, D.object_light, D.n_objects, &d.obj_light, "object lights");
    if (!rc) rc = upload(ctx, s, D.materials, D.n_materials, &d.mats, "materials");
    if (!rc) rc = upload(ctx, s, D.spectra, D.n_spectra, &d.specs, "spectra");
    if (!rc) rc = upload(ctx, s, D.spectrum_pool, D.pool_size, &d.pool, "spectrum pool");
    if (!rc) rc = upload(ctx, s, spec_max.data(), spec_max.size(), &d.spec_max, "spectrum maxima");
    if (!rc) rc = upload(ctx, s, D.lights, D.n_lights, &d.lights, "lights");
    if (!rc) rc = upload(ctx, s, cdf.data(), cdf.size(), &d.light_cdf, "light cdf");
    if (!rc) rc = upload(ctx, s, area.data(), area.size(), &d.light_area, "light areas");
    if (!rc) rc = upload(ctx, s, tri_cdf.data(), tri_cdf.size(), &d.tri_cdf, "mesh light cdf");
    if (!rc) rc = upload(ctx, s, ow.data(), no, &d.obs_w, "observer");
    if (!rc) rc = upload(ctx, s, oxyz.data(), 3 * no, &d.obs_xyz, "observer");
    if (!rc) rc = upload(ctx, s, odxyz.data(), 3 * no, &d.obs_dxyz, "observer");
    if (!rc) rc = upload(ctx, s, ocdf.data(), no, &d.obs_cdf, "observer");
    if (rc) {
        liar_gpu_scene_destroy(s);
        return rc;
    }
    s->h_lights.assign(D.lights, D.lights + D.n_lights);
    s->h_materials.assign(D.materials, D.materials + D.n_materials);
    d.nodes = mesh_nodes(s->mesh);
    d.qtris = mesh_tris(s->mesh);
    d.n_lights = (int)D.n_lights;
    d.n_tex = (int)D.n_textures;
    d.n_obs = (int)no;
    d.sky_light = sky;
    // LightSky::doSetSceneBound: intersections with the sky lie 1000 scene radii away
    d.sky_distance = D.scene_radius > 0 ? 1e3f * D.scene_radius : 1e3f;
    d.stack_needed = mesh_stack_needed(s->mesh);
    {
        // the description's own device copy, which out-of-line device code reads it through
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, sizeof(DScene));
        if (e == cudaSuccess) {
            s->buffers.push_back(p);
            d.self = static_cast<const DScene*>(p);
            e = cudaMemcpy(p, &d, sizeof(DScene), cudaMemcpyHostToDevice);
        }
        if (e != cudaSuccess) {
            cudaGetLastError();
            const int r = ctx_cuda(ctx, e, "scene description");
            liar_gpu_scene_destroy(s);
            return r;
        }
    }
    s->n_triangles = D.n_triangles;
    *out = s;
    return LIAR_OK;
}

namespace liar_gpu {
namespace rt {
// accessors for the other subsystems that shade against an uploaded scene (photon tracing)
const DScene& scene_dscene(const liar_gpu_scene* s) { return s->d; }
const std::vector<liar_light>& scene_lights(const liar_gpu_scene* s) { return s->h_lights; }
const std::vector<liar_material>& scene_materials(const liar_gpu_scene* s) { return s->h_materials; }
unsigned long long* render_stats_device(liar_gpu_ctx* ctx, cudaStream_t st) {
    RenderBuffers* rb = render_buffers(ctx);
    if (!rb->stats && ensure_render_buffers(ctx, rb, 0)) return nullptr;
    return rb->stats;
}
const liar_gpu_mesh* scene_mesh(const liar_gpu_scene* s) { return s->mesh; }
int scene_device(const liar_gpu_scene* s) { return s->device; }
uint64_t scene_uid(const liar_gpu_scene* s) { return s->uid; }
}  // namespace rt
}  // namespace liar_gpu

extern "C" void liar_gpu_scene_destroy(liar_gpu_scene* s) {
    if (!s) return;
    int cur = -1;
    cudaGetDevice(&cur);
    if (s->device >= 0) cudaSetDevice(s->device);
    for (void* p : s->buffers) cudaFree(p);
    if (s->mesh) liar_gpu_mesh_destroy(s->mesh);
    if (cur >= 0) cudaSetDevice(cur);
    delete s;
}

namespace liar_gpu {
namespace rt {
// PhotonMapper (photon_mapper.cu): photon maps, then the DirectLighting wavefront with their estimates
int render_photon_mapper(liar_gpu_ctx* ctx, const liar_gpu_scene* scene, const liar_render_desc& R, float* d_film,
                         cudaStream_t st);
}  // namespace rt
}  // namespace liar_gpu

namespace {

int render_impl(liar_gpu_ctx* ctx, const liar_gpu_scene* scene, const liar_render_desc* desc, float* d_film,
                cudaStream_t st) {
    const liar_render_desc& R = *desc;
    if (R.width <= 0 || R.height <= 0 || R.spp <= 0) return ctx_fail(ctx, LIAR_ERR_INVALID, "empty image or no samples");
    if (R.max_ray_generation < 0) return ctx_fail(ctx, LIAR_ERR_INVALID, "max_ray_generation must be >= 0");
    if (const char* m = film_desc_error(R)) return ctx_fail(ctx, LIAR_ERR_INVALID, "%s", m);
    if (R.sampler & ~(LIAR_SAMPLER_LATIN_HYPERCUBE | LIAR_SAMPLER_NOT_JITTERED))
        return ctx_fail(ctx, LIAR_ERR_INVALID, "unknown sampler bits 0x%x", (unsigned)R.sampler);
    if (R.tracer == LIAR_TRACER_DIRECT_LIGHTING) return render_direct(ctx, scene, R, d_film, st, nullptr);
    if (R.tracer == LIAR_TRACER_PHOTON_MAPPER) return render_photon_mapper(ctx, scene, R, d_film, st);
    if (R.tracer != LIAR_TRACER_ADJOINT_PHOTON) return ctx_fail(ctx, LIAR_ERR_UNSUPPORTED, "tracer %d", R.tracer);
    const uint64_t total = (uint64_t)R.width * R.height * R.spp;
    if ((uint64_t)R.width * R.height >= (1ull << 32)) return ctx_fail(ctx, LIAR_ERR_INVALID, "image too large");
    uint64_t wave = R.wave_paths > 0 ? (uint64_t)R.wave_paths : (1ull << 22);
    if (wave > total) wave = total;
    RenderBuffers* rb = render_buffers(ctx);
    int rc = ensure_render_buffers(ctx, rb, (size_t)wave);
    if (rc) return rc;
    cudaError_t e = cudaMemsetAsync(rb->stats, 0, 4 * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "reset statistics");
    WaveParams W;
    W.cam = R.camera;
    W.width = R.width;
    W.height = R.height;
    W.spp = R.spp;
    W.max_gen = R.max_ray_generation;
    W.max_depth = R.max_depth;
    W.sampler = (uint32_t)R.sampler;
    W.seed = mix64(R.seed ^ mix64(0x51ed270b27ad0e0dull + (uint64_t)(uint32_t)R.first_sample));
    W.film = film_spec(d_film, R);
    const DScene& S = scene->d;
    for (uint64_t first = 0; first < total; first += wave) {
        if (ctx_cancel_requested(ctx)) return ctx_cancelled(ctx, st);
        const uint32_t n = (uint32_t)std::min<uint64_t>(wave, total - first);
        W.first_path = first;
        int cur = 0;
        e = cudaMemsetAsync(rb->q[0].count, 0, 4, st);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "reset queue");
        k_raygen<<<(n + 255) / 256, 256, 0, st>>>(S, W, rb->P, rb->q[0], n, rb->stats);
        // Bounce b reads queue c_b and writes c_{b+1} <= c_b. The host launches bounce b sized for
        // c_{b-1}, the kernels read c_b on the device, and the host waits for c_b only after
        // bounce b is queued, so the GPU never idles on the round trip; the bounce launched
        // after the last non-empty one finds an empty queue and ends at once.
        uint32_t bound = n;  // c_{b-1}: an upper bound of the queue bounce b reads
        for (int bounce = 0; bound > 0; ++bounce) {
            if (bounce > 4096) return ctx_fail(ctx, LIAR_ERR_TIMEOUT, "paths did not terminate after 4096 bounces");
            if (ctx_cancel_requested(ctx)) return ctx_cancelled(ctx, st);
            const uint32_t* n_dev = bounce == 0 ? nullptr : rb->q[cur].count;
            rc = trace_mesh_internal(ctx, scene->mesh, rb->q[cur].rays, bound, rb->hits, 0, st, kCounterWord + 8, n_dev);
            if (rc) return rc;
            e = cudaMemsetAsync(rb->q[cur ^ 1].count, 0, 4, st);
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "reset queue");
            (S.n_tex > 0 ? k_shade<true> : k_shade<false>)<<<(bound + 127) / 128, 128, 0, st>>>(
                S, W, rb->P, rb->q[cur], rb->hits, bound, n_dev, rb->q[cur ^ 1], rb->stats);
            e = cudaGetLastError();
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "shade launch");
            cur ^= 1;
            const int slot = (bounce + 1) & 1;  // c_{b+1}
            e = cudaMemcpyAsync(rb->h_count + slot, rb->q[cur].count, 4, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaEventRecord(rb->ev[slot], st);
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "queue size");
            if (bounce == 0) continue;  // c_0 = n is known: bounce 1 is launched for n
            // c_b, copied after bounce b - 1, bounds bounce b + 1
            e = cudaEventSynchronize(rb->ev[bounce & 1]);
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "queue size");
            bound = rb->h_count[bounce & 1];
        }
    }
    // path count
    unsigned long long paths = total;
    e = cudaMemcpyAsync(rb->stats, &paths, sizeof(paths), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "statistics");
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "render synchronize");
    return ctx_check_status(ctx);
}

}  // namespace

extern "C" int liar_gpu_render_device(liar_gpu_ctx* ctx, const liar_gpu_scene* scene, const liar_render_desc* desc,
                                      float* d_film, void* stream) {
    if (!ctx) return LIAR_ERR_INVALID;
    if (!scene || !desc || !d_film) return ctx_fail(ctx, LIAR_ERR_INVALID, "null scene, description or film");
    if (scene->device != ctx->device) return ctx_fail(ctx, LIAR_ERR_INVALID, "scene lives on another device");
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    return render_impl(ctx, scene, desc, d_film, stream ? (cudaStream_t)stream : ctx->stream);
}

extern "C" int liar_gpu_render(liar_gpu_ctx* ctx, const liar_gpu_scene* scene, const liar_render_desc* desc,
                               float* film) {
    if (!ctx) return LIAR_ERR_INVALID;
    if (!scene || !desc || !film) return ctx_fail(ctx, LIAR_ERR_INVALID, "null scene, description or film");
    if (desc->width <= 0 || desc->height <= 0) return ctx_fail(ctx, LIAR_ERR_INVALID, "empty image");
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    const size_t bytes = (size_t)desc->width * desc->height * 8 * sizeof(float);
    float* d_film = nullptr;
    cudaError_t e = cudaMalloc((void**)&d_film, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return ctx_cuda(ctx, e, "film");
    }
    e = cudaMemcpyAsync(d_film, film, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) rc = render_impl(ctx, scene, desc, d_film, ctx->stream);
    else rc = ctx_cuda(ctx, e, "film copy in");
    if (!rc || rc == LIAR_ERR_CANCELLED) {  // a cancelled render hands back its partial film
        e = cudaMemcpyAsync(film, d_film, bytes, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = ctx_cuda(ctx, e, "film copy out");
    }
    cudaFree(d_film);
    return rc;
}

extern "C" int liar_gpu_render_stats(const liar_gpu_ctx* ctx, unsigned long long* out3) {
    if (!ctx || !out3) return LIAR_ERR_INVALID;
    for (auto& ext : ctx->extensions)
        if (ext.first == "render") {
            RenderBuffers* rb = static_cast<RenderBuffers*>(ext.second);
            if (!rb->stats) break;
            if (cudaMemcpy(out3, rb->stats, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost) != cudaSuccess) {
                cudaGetLastError();
                return LIAR_ERR_CUDA;
            }
            return LIAR_OK;
        }
    out3[0] = out3[1] = out3[2] = 0;
    return LIAR_OK;
}
