// batch.cu -- many scenes in one CUDA-graph launch (no reference counterpart: the reference renders
// one scene per process, src/liar/kernel/render_engine.cpp:170-358).
//
// Each item (scene, camera, resolution, spp) owns a contiguous range of one global path index
// space. The graph holds a WHILE conditional node; each iteration renders one wave of that space:
//   raygen  -> [memset counter, trace (scene table), memset queue, shade] x max_bounces -> wave_end
// wave_end advances the wave counter and sets the loop condition on the device, so a whole batch
// is a single cudaGraphLaunch. Queue sizes never leave the device: the trace kernel reads its
// ray count from device memory and the raygen / shade kernels are grid-stride over device counts.
// The shading is the AdjointPhotonTracer estimator of render.cu (one-sample MIS, RR, emission on
// light hits) with an optional hero-wavelength spectral estimator (Wilkie et al. 2014).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "../../include/liar_gpu.h"
#include "ctx.h"
#include "render_dev.cuh"
#include "traverse.cuh"

using namespace liar_gpu;
using namespace liar_gpu::rt;

namespace liar_gpu {
namespace rt {
const DScene& scene_dscene(const liar_gpu_scene* s);
const liar_gpu_mesh* scene_mesh(const liar_gpu_scene* s);
int scene_device(const liar_gpu_scene* s);
}  // namespace rt
}  // namespace liar_gpu

namespace {

struct BItem {
    int scene;
    int width, height, spp, max_gen, max_depth;
    uint32_t sampler;  // SAMPLER_* mode bits (sampler.h)
    uint64_t seed;
    uint64_t path_begin;
    FilmSpec film;
    liar_camera cam;
};

struct BControl {
    uint32_t wave;
    uint32_t n_waves;
    uint32_t count[2];  // queue sizes
    uint32_t work;      // trace work counter
    uint32_t pad[3];
    unsigned long long stats[4];  // paths, segments, hits, waves
};

template <int H>
struct BState {
    int32_t* item;
    float* lam;      // H per path
    float* T;        // H per path
    float* L;        // H per path
    float* pdfsum;   // sum of the observer pdf over the hero wavelengths
    float* alpha;
    int32_t* gen;
};

struct BQueue {
    liar_ray* rays;
    uint32_t* slot;
    uint32_t* scene;
};

struct BParams {
    const DScene* scenes;
    const BItem* items;
    const uint64_t* item_begin;  // n_items + 1
    int n_items;
    uint64_t total_paths;
    uint32_t wave_paths;
    BControl* ctrl;
};

__device__ __forceinline__ int find_item(const uint64_t* begin, int n, uint64_t g) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (begin[mid] <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ float observer_pdf(const DScene& S, float w) {
    const int i = upper_bound_f(S.obs_w, S.n_obs, w);
    if (i == 0 || i == S.n_obs) return 0.0f;
    return (S.obs_cdf[i] - S.obs_cdf[i - 1]) / (S.obs_w[i] - S.obs_w[i - 1]);
}

// the hero wavelengths: lam[0] sampled, the others rotated by a quarter of the observer range
template <int H>
__device__ __forceinline__ void hero_wavelengths(const DScene& S, float u, float* lam, float& pdfsum) {
    float pdf0;
    lam[0] = observer_sample(S, u, pdf0);
    if (H == 1) {
        pdfsum = pdf0;
        return;
    }
    const float w0 = S.obs_w[0], range = S.obs_w[S.n_obs - 1] - w0;
    pdfsum = pdf0;
    for (int i = 1; i < H; ++i) {
        float x = (lam[0] - w0) + range * ((float)i / (float)H);
        if (x >= range) x -= range;
        lam[i] = w0 + x;
        pdfsum += observer_pdf(S, lam[i]);
    }
    if (!(pdf0 > 0.0f)) pdfsum = 0.0f;
}

__device__ __forceinline__ void bqueue_push(const BQueue& q, uint32_t* count, bool want, const liar_ray& r, uint32_t slot,
                                            uint32_t scene) {
    const uint32_t mask = __ballot_sync(0xffffffffu, want);
    if (mask == 0) return;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(count, (uint32_t)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (want) {
        const uint32_t s = base + __popc(mask & ((1u << lane) - 1u));
        float4* dst = reinterpret_cast<float4*>(q.rays + s);
        dst[0] = make_float4(r.ox, r.oy, r.oz, r.tmin);
        dst[1] = make_float4(r.dx, r.dy, r.dz, r.tmax);
        q.slot[s] = slot;
        q.scene[s] = scene;
    }
}

template <int H>
__device__ void bsplat(const DScene& S, const BItem& it, uint64_t local, const float* lam, const float* L, float pdfsum,
                       float alpha) {
    float3 xyz = mk(0, 0, 0);
    if (pdfsum > 0.0f) {
        // balance heuristic over the hero rotations: sum_i L(lam_i) cmf(lam_i) / sum_k p(lam_k)
        for (int i = 0; i < H; ++i) {
            const float3 c = observer_sensitivity(S, lam[i]);
            const float s = L[i] / pdfsum;
            xyz = xyz + mk(s * c.x, s * c.y, s * c.z);
        }
    }
    SampleKey k;
    k.seed = it.seed;
    k.pixel = (uint32_t)(local / (uint64_t)it.spp);
    k.sample = (uint32_t)(local % (uint64_t)it.spp);
    k.spp = (uint32_t)it.spp;
    k.mode = it.sampler;
    film_splat(it.film, k, xyz, alpha);
}

template <int H>
__global__ void __launch_bounds__(256) k_b_raygen(BParams P, BState<H> st, BQueue out) {
    BControl* C = P.ctrl;
    const uint64_t base = (uint64_t)C->wave * P.wave_paths;
    const uint64_t n64 = base < P.total_paths ? std::min<uint64_t>(P.wave_paths, P.total_paths - base) : 0;
    const uint32_t n = (uint32_t)n64;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t b0 = blockIdx.x * blockDim.x; b0 < n; b0 += stride) {
        const uint32_t i = b0 + threadIdx.x;
        bool want = false;
        liar_ray r{};
        uint32_t sc = 0;
        if (i < n) {
            const uint64_t g = base + i;
            const int ii = find_item(P.item_begin, P.n_items, g);
            const BItem it = P.items[ii];
            const DScene& S = P.scenes[it.scene];
            const uint64_t local = g - it.path_begin;
            SampleKey k;
            k.seed = it.seed;
            k.pixel = (uint32_t)(local / (uint64_t)it.spp);
            k.sample = (uint32_t)(local % (uint64_t)it.spp);
            k.spp = (uint32_t)it.spp;
            k.mode = it.sampler;
            float lam[H], pdfsum;
            hero_wavelengths<H>(S, sample_dim(k, DIM_LAMBDA, true), lam, pdfsum);
            r = camera_ray(it.cam, k, it.width, it.height);
            st.item[i] = ii;
            for (int h = 0; h < H; ++h) {
                st.lam[(size_t)H * i + h] = lam[h];
                st.T[(size_t)H * i + h] = 1.0f;
                st.L[(size_t)H * i + h] = 0.0f;
            }
            st.pdfsum[i] = pdfsum;
            st.alpha[i] = 0.0f;
            st.gen[i] = 0;
            sc = (uint32_t)it.scene;
            want = true;
        }
        bqueue_push(out, &C->count[0], want, r, i, sc);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&C->stats[0], (unsigned long long)n);
}

template <int H, bool TEX>
__global__ void __launch_bounds__(128) k_b_shade(BParams P, BState<H> st, BQueue in, const liar_hit* __restrict__ hits,
                                                 int cur, BQueue out) {
    BControl* C = P.ctrl;
    const uint32_t n_in = C->count[cur];
    const uint32_t stride = gridDim.x * blockDim.x;
    unsigned long long segs = 0, n_hit = 0;
    for (uint32_t b0 = blockIdx.x * blockDim.x; b0 < n_in; b0 += stride) {
        const uint32_t q = b0 + threadIdx.x;
        bool want = false;
        liar_ray nr{};
        uint32_t p = 0, sc = 0;
        if (q < n_in) {
            ++segs;
            p = in.slot[q];
            const int ii = st.item[p];
            const BItem& it = P.items[ii];
            const DScene& S = P.scenes[it.scene];
            sc = (uint32_t)it.scene;
            const float4 r0 = reinterpret_cast<const float4*>(in.rays + q)[0];
            const float4 r1 = reinterpret_cast<const float4*>(in.rays + q)[1];
            const float3 o = mk(r0.x, r0.y, r0.z), d = mk(r1.x, r1.y, r1.z);
            const liar_hit h = hits[q];
            const uint64_t g = (uint64_t)C->wave * P.wave_paths + p;
            const uint64_t local = g - it.path_begin;
            SampleKey key;
            key.seed = it.seed;
            key.pixel = (uint32_t)(local / (uint64_t)it.spp);
            key.sample = (uint32_t)(local % (uint64_t)it.spp);
            key.spp = (uint32_t)it.spp;
            key.mode = it.sampler;
            // low 16 bits: ray generation; bit 16: the path crossed a dispersive interface and
            // carries lam[0] alone
            const int gen_word = st.gen[p];
            const int gen = gen_word & 0xffff;
            bool single = (gen_word >> 16) & 1;
            float T[H], L[H], lam[H];
            for (int k = 0; k < H; ++k) {
                T[k] = st.T[(size_t)H * p + k];
                L[k] = st.L[(size_t)H * p + k];
                lam[k] = st.lam[(size_t)H * p + k];
            }
            bool alive = false;
            float3 next_o = mk(0, 0, 0), next_d = mk(0, 0, 1);
            float next_tmin = kTol, next_tmax = INFINITY;
            if (h.prim < 0) {
                if (S.sky_light >= 0 && S.sky_distance > r0.w * (1.0f + kTol) && S.sky_distance < r1.w * (1.0f - kTol)) {
                    if (gen == 0) st.alpha[p] = 1.0f;
                    if (gen > 0)
                        for (int k = 0; k < H; ++k) L[k] += T[k] * spec_eval(S, S.lights[S.sky_light].spectrum, lam[k], false);
                }
            } else {
                ++n_hit;
                if (gen == 0) st.alpha[p] = 1.0f;
                HitContext HC = hit_context(S, o, d, (uint32_t)h.prim, h.t);
                // the camera vertex carries the camera's ray differentials (texture filtering)
                if (S.n_tex > 0 && gen == 0) camera_footprint(S, HC, (uint32_t)h.prim, it.cam, key, it.width, it.height);
                const int light = HC.light, mi = HC.mat;
                if (gen > 0 && light >= 0)
                    for (int k = 0; k < H; ++k) L[k] += T[k] * spec_eval(S, S.lights[light].spectrum, lam[k], false);
                const bool shader_emits = gen == 0 || light < 0;  // as render.cu
                if (mi < 0) {
                    alive = true;
                    next_o = o;
                    next_d = d;
                    next_tmin = h.t + kTol;
                    next_tmax = r1.w;
                } else if (S.mats[mi].type == LIAR_MAT_NONE) {
                    if (shader_emits && S.mats[mi].emission >= 0)
                        for (int k = 0; k < H; ++k) L[k] += T[k] * spec_eval(S, S.mats[mi].emission, lam[k], false);
                } else {
                    const liar_material M = S.mats[mi];
                    if (shader_emits && M.emission >= 0)
                        for (int k = 0; k < H; ++k) L[k] += T[k] * spec_eval(S, M.emission, lam[k], false);
                    const Bsdf B = make_bsdf<TEX>(S, M, HC, lam[0]);
                    const float3 md = -d;
                    float3 wi = mk(dot(md, HC.u), dot(md, HC.v), dot(md, HC.N));
                    wi.z = fmaxf(wi.z, kEps);
                    const bool strat = gen < it.max_gen;
                    const uint32_t base = DIM_GEN0 + DIMS_PER_GEN * (uint32_t)gen;
                    const float spdf = (has_caps(B.caps, CAP_DIFF) || has_caps(B.caps, CAP_GLOSSY)) ? 0.5f : 1.0f;
                    float3 wo = mk(0, 0, 1);
                    float w_mis = 0.0f, pdf = 0.0f;
                    bool ok = false;
                    bool from_bsdf = false;
                    BsdfSample bs{mk(0, 0, 0), 0.0f, 0.0f};
                    if (sample_dim(key, base + OFF_STRATEGY, strat) < spdf) {
                        bs = bsdf_sample(B, wi, sample_dim(key, base + OFF_BSDF, strat),
                                         sample_dim(key, base + OFF_BSDF + 1, strat),
                                         sample_dim(key, base + OFF_COMPONENT, strat), CAP_ALL);
                        if (bs.ok()) {
                            pdf = bs.pdf * spdf;
                            const float3 wd = bs.wo.x * HC.u + bs.wo.y * HC.v + bs.wo.z * HC.N;
                            float pl = 0.0f;
                            for (int l = 0; l < S.n_lights; ++l) {
                                const LightEmission e = light_emission(S, l, HC.target, wd, lam[0]);
                                if (e.pdf > 0.0f) pl += light_choice_pdf(S, l) * e.pdf;
                            }
                            pl *= (1.0f - spdf);
                            w_mis = power_heuristic(pdf, pl);
                            wo = bs.wo;
                            ok = true;
                            from_bsdf = true;
                        }
                    } else if (S.n_lights > 0) {
                        const float uc = sample_dim(key, base + OFF_LIGHT_CHOICE, strat);
                        int kk = lower_bound_f(S.light_cdf, S.n_lights, uc);
                        if (kk > S.n_lights - 1) kk = S.n_lights - 1;
                        const float pc = light_choice_pdf(S, kk);
                        if (pc > 0.0f) {
                            const LightSample ls = light_sample(S, kk, HC.target, sample_dim(key, base + OFF_LIGHT, strat),
                                                                sample_dim(key, base + OFF_LIGHT + 1, strat), lam[0]);
                            if (ls.pdf > 0.0f) {
                                float lp = pc * ls.pdf;
                                for (int l = 0; l < S.n_lights; ++l) {
                                    if (l == kk) continue;
                                    const LightEmission e = light_emission(S, l, HC.target, ls.dir, lam[0]);
                                    if (e.pdf > 0.0f) lp += light_choice_pdf(S, l) * e.pdf;
                                }
                                lp *= (1.0f - spdf);
                                const float3 lwo = mk(dot(ls.dir, HC.u), dot(ls.dir, HC.v), dot(ls.dir, HC.N));
                                const BsdfOut be = bsdf_evaluate(B, wi, lwo, CAP_ALL);
                                if (be.pdf > 0.0f && be.value != 0.0f) {
                                    wo = lwo;
                                    pdf = lp;
                                    w_mis = power_heuristic(lp, be.pdf * spdf);
                                    ok = true;
                                }
                            }
                        }
                    }
                    if (ok) {
                        // the BSDF value at every hero wavelength along the chosen direction
                        const bool dispersive = (M.type == LIAR_MAT_DIELECTRIC || M.type == LIAR_MAT_WALTER) &&
                                                (M.tex[0] >= 0 || M.tex[1] >= 0 ||
                                                 (M.spec[0] >= 0 && S.specs[M.spec[0]].type != LIAR_SPEC_CONSTANT) ||
                                                 (M.spec[1] >= 0 && S.specs[M.spec[1]].type != LIAR_SPEC_CONSTANT));
                        float val[H];
                        for (int k = 0; k < H; ++k) {
                            if (k > 0 && dispersive) {
                                val[k] = 0.0f;  // secondary wavelengths end at a dispersive interface
                                continue;
                            }
                            const Bsdf Bk = k == 0 ? B : make_bsdf<TEX>(S, M, HC, lam[k]);
                            if (from_bsdf) {
                                if (k == 0) {
                                    val[k] = bs.value;
                                } else if (Bk.type == LIAR_MAT_CONDUCTOR) {
                                    val[k] = Bk.r * fresnel_conductor(Bk.eta, Bk.kappa, wi.z) / wi.z;
                                } else if (Bk.type == LIAR_MAT_MIRROR) {
                                    val[k] = Bk.r;
                                } else if (Bk.type == LIAR_MAT_DIELECTRIC) {
                                    // constant index: same Fresnel, only the reflectance / transmittance differ
                                    val[k] = wo.z > 0.0f ? bs.value * (B.r != 0.0f ? Bk.r / B.r : 0.0f)
                                                         : bs.value * (B.t != 0.0f ? Bk.t / B.t : 0.0f);
                                } else {
                                    val[k] = bsdf_do_evaluate(Bk, wi, wo, CAP_ALL).value;
                                }
                            } else {
                                val[k] = bsdf_evaluate(Bk, wi, wo, CAP_ALL).value;
                            }
                        }
                        const float cos_t = wo.z;
                        next_o = HC.target + ((cos_t > 0.0f ? 10.0f : -10.0f) * kTol) * HC.ng;
                        next_d = wo.x * HC.u + wo.y * HC.v + wo.z * HC.N;
                        next_tmin = kTol;
                        next_tmax = INFINITY;
                        float f = w_mis * (fabsf(cos_t) / pdf);
                        if (H > 1 && dispersive && !single) {
                            // from here on the path exists for lam[0] alone: its later radiance is
                            // weighted by 1 / p(lam[0]) instead of the hero sum 1 / sum_k p(lam[k])
                            // (the splat divides by the sum; radiance gathered so far keeps it)
                            const float p0 = observer_pdf(S, lam[0]);
                            f = p0 > 0.0f ? f * (st.pdfsum[p] / p0) : 0.0f;
                            single = true;
                        }
                        for (int k = 0; k < H; ++k) T[k] *= val[k] * f;
                        alive = true;
                    }
                }
            }
            if (alive) {
                const int ng1 = gen + 1;
                if (it.max_depth > 0 && ng1 >= it.max_depth) {
                    alive = false;
                } else if (ng1 >= it.max_gen) {
                    const float ur = sample_dim(key, DIM_GEN0 + DIMS_PER_GEN * (uint32_t)ng1 + OFF_RR, false);
                    if (ur < 0.5f)
                        for (int k = 0; k < H; ++k) T[k] /= 0.5f;
                    else
                        alive = false;
                }
            }
            if (alive) {
                for (int k = 0; k < H; ++k) {
                    st.T[(size_t)H * p + k] = T[k];
                    st.L[(size_t)H * p + k] = L[k];
                }
                st.gen[p] = (gen + 1) | (single ? 0x10000 : 0);
                nr = liar_ray{next_o.x, next_o.y, next_o.z, next_tmin, next_d.x, next_d.y, next_d.z, next_tmax};
                want = true;
            } else {
                bsplat<H>(S, it, local, lam, L, st.pdfsum[p], st.alpha[p]);
            }
        }
        bqueue_push(out, &C->count[cur ^ 1], want, nr, p, sc);
    }
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        segs += __shfl_down_sync(0xffffffffu, segs, o);
        n_hit += __shfl_down_sync(0xffffffffu, n_hit, o);
    }
    if (lane == 0 && segs) {
        atomicAdd(&C->stats[1], segs);
        atomicAdd(&C->stats[2], n_hit);
    }
}

// paths still queued after the last unrolled bounce end here (their gathered radiance counts)
template <int H>
__global__ void __launch_bounds__(256) k_b_flush(BParams P, BState<H> st, BQueue in, int cur) {
    BControl* C = P.ctrl;
    const uint32_t n = C->count[cur];
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const uint32_t p = in.slot[q];
        const BItem& it = P.items[st.item[p]];
        const uint64_t g = (uint64_t)C->wave * P.wave_paths + p;
        float lam[H], L[H];
        for (int k = 0; k < H; ++k) {
            lam[k] = st.lam[(size_t)H * p + k];
            L[k] = st.L[(size_t)H * p + k];
        }
        bsplat<H>(P.scenes[it.scene], it, g - it.path_begin, lam, L, st.pdfsum[p], st.alpha[p]);
    }
}

__global__ void k_b_clear_queue(BControl* C, int which) { C->count[which] = 0; }
__global__ void k_b_clear_work(BControl* C) { C->work = 0; }

__global__ void k_b_wave_end(BControl* C, cudaGraphConditionalHandle handle) {
    C->wave += 1;
    C->stats[3] += 1;
    cudaGraphSetConditional(handle, C->wave < C->n_waves ? 1u : 0u);
}

__global__ void k_b_begin(BControl* C, uint32_t n_waves) {
    C->wave = 0;
    C->n_waves = n_waves;
    C->count[0] = C->count[1] = 0;
    C->work = 0;
    C->stats[0] = C->stats[1] = C->stats[2] = C->stats[3] = 0;
}

}  // namespace

struct liar_gpu_batch {
    int device = -1;
    int hero = 1;
    int bounces = 8;
    uint32_t wave = 0;
    uint32_t n_waves = 0;
    uint64_t total = 0;
    int shade_blocks_per_sm = 16;
    bool textured = false;  // some scene has textures: the shading kernel with texture lookups
    liar_trace_config trace{128, 16};
    std::vector<void*> buffers;
    BParams params{};
    BControl* ctrl = nullptr;
    TreeRoot* roots = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned long long h_stats[4] = {0, 0, 0, 0};
};

namespace {

int b_alloc(liar_gpu_ctx* ctx, liar_gpu_batch* b, size_t bytes, void** p, const char* what) {
    cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return ctx_cuda(ctx, e, what);
    }
    b->buffers.push_back(*p);
    return LIAR_OK;
}

struct TraceLaunch {
    const void* kern;
    size_t smem;
    unsigned grid;
    int block;
};

// kernel choice, shared memory attribute and occupancy, all resolved before stream capture
int trace_launch_shape(liar_gpu_ctx* ctx, const liar_trace_config& cfg, TraceLaunch& tl) {
    const int S = cfg.smem_stack, BL = cfg.block_size;
    if (S == 8 && BL == 128) tl.kern = (const void*)trace_multi_kernel<8, 128>;
    else if (S == 16 && BL == 128) tl.kern = (const void*)trace_multi_kernel<16, 128>;
    else if (S == 24 && BL == 128) tl.kern = (const void*)trace_multi_kernel<24, 128>;
    else if (S == 8 && BL == 256) tl.kern = (const void*)trace_multi_kernel<8, 256>;
    else if (S == 16 && BL == 256) tl.kern = (const void*)trace_multi_kernel<16, 256>;
    else return ctx_fail(ctx, LIAR_ERR_INVALID, "no trace kernel for block %d, shared stack %d", BL, S);
    tl.smem = (size_t)S * BL * 8;
    tl.block = BL;
    cudaError_t e = cudaFuncSetAttribute(tl.kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tl.smem);
    int per_sm = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tl.kern, BL, tl.smem);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "batch trace set-up");
    tl.grid = (unsigned)(ctx->num_sms * std::max(per_sm, 1));
    return LIAR_OK;
}

template <int H>
int capture_body(liar_gpu_ctx* ctx, liar_gpu_batch* b, cudaStream_t cs, BState<H> st, BQueue* q, liar_hit* hits,
                 cudaGraphConditionalHandle handle, const TraceLaunch& tl) {
    const BParams& P = b->params;
    const int sms = ctx->num_sms;
    k_b_clear_queue<<<1, 1, 0, cs>>>(b->ctrl, 0);
    k_b_raygen<H><<<sms * 8, 256, 0, cs>>>(P, st, q[0]);
    int cur = 0;
    for (int bounce = 0; bounce < b->bounces; ++bounce) {
        k_b_clear_work<<<1, 1, 0, cs>>>(b->ctrl);
        // trace the current queue (ray count read on the device)
        const uint32_t* n_dev = &b->ctrl->count[cur];
        uint32_t* work = &b->ctrl->work;
        uint32_t* status = ctx->d_scratch + kStatusWord;
        void* args[] = {(void*)&b->roots, (void*)&q[cur].rays, (void*)&q[cur].scene, (void*)&hits,
                        (void*)&n_dev, (void*)&work, (void*)&status};
        cudaError_t e = cudaLaunchKernel(tl.kern, dim3(tl.grid), dim3(tl.block), args, tl.smem, cs);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "batch trace launch");
        k_b_clear_queue<<<1, 1, 0, cs>>>(b->ctrl, cur ^ 1);
        (b->textured ? k_b_shade<H, true> : k_b_shade<H, false>)<<<sms * b->shade_blocks_per_sm, 128, 0, cs>>>(P, st, q[cur], hits, cur, q[cur ^ 1]);
        cur ^= 1;
    }
    k_b_flush<H><<<sms * 4, 256, 0, cs>>>(P, st, q[cur], cur);
    k_b_wave_end<<<1, 1, 0, cs>>>(b->ctrl, handle);
    return ctx_cuda(ctx, cudaGetLastError(), "batch capture");
}

template <int H>
int build_graph(liar_gpu_ctx* ctx, liar_gpu_batch* b) {
    const size_t W = b->params.wave_paths;
    BState<H> st;
    BQueue q[2];
    liar_hit* hits = nullptr;
    void* p = nullptr;
    int rc = b_alloc(ctx, b, W * (4 + 3 * 4 * H + 4 + 4 + 4), &p, "batch path state");
    if (rc) return rc;
    char* c = static_cast<char*>(p);
    st.item = reinterpret_cast<int32_t*>(c);
    c += W * 4;
    st.lam = reinterpret_cast<float*>(c);
    c += W * 4 * H;
    st.T = reinterpret_cast<float*>(c);
    c += W * 4 * H;
    st.L = reinterpret_cast<float*>(c);
    c += W * 4 * H;
    st.pdfsum = reinterpret_cast<float*>(c);
    c += W * 4;
    st.alpha = reinterpret_cast<float*>(c);
    c += W * 4;
    st.gen = reinterpret_cast<int32_t*>(c);
    for (int k = 0; k < 2; ++k) {
        rc = b_alloc(ctx, b, W * sizeof(liar_ray), &p, "batch queue");
        if (rc) return rc;
        q[k].rays = static_cast<liar_ray*>(p);
        rc = b_alloc(ctx, b, W * 8, &p, "batch queue");
        if (rc) return rc;
        q[k].slot = static_cast<uint32_t*>(p);
        q[k].scene = static_cast<uint32_t*>(p) + W;
    }
    rc = b_alloc(ctx, b, W * sizeof(liar_hit), &p, "batch hits");
    if (rc) return rc;
    hits = static_cast<liar_hit*>(p);

    TraceLaunch tl;
    rc = trace_launch_shape(ctx, b->trace, tl);
    if (rc) return rc;
    cudaError_t e = cudaGraphCreate(&b->graph, 0);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "graph create");
    cudaGraphConditionalHandle handle;
    e = cudaGraphConditionalHandleCreate(&handle, b->graph, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "conditional handle");
    // begin node: reset the control block
    cudaKernelNodeParams kp = {};
    void* begin_args[] = {(void*)&b->ctrl, (void*)&b->n_waves};
    kp.func = (void*)k_b_begin;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(1);
    kp.kernelParams = begin_args;
    cudaGraphNode_t begin_node;
    e = cudaGraphAddKernelNode(&begin_node, b->graph, nullptr, 0, &kp);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "graph begin node");
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t loop_node;
    e = cudaGraphAddNode(&loop_node, b->graph, &begin_node, 1, &cp);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "graph while node");
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    cudaStream_t cs;
    e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "capture stream");
    e = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaStreamDestroy(cs);
        return ctx_cuda(ctx, e, "begin capture");
    }
    rc = capture_body<H>(ctx, b, cs, st, q, hits, handle, tl);
    cudaGraph_t captured = nullptr;
    e = cudaStreamEndCapture(cs, &captured);
    cudaStreamDestroy(cs);
    if (rc) return rc;
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "end capture");
    e = cudaGraphInstantiate(&b->exec, b->graph, 0);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "graph instantiate");
    return LIAR_OK;
}

}  // namespace

extern "C" int liar_gpu_batch_create(liar_gpu_ctx* ctx, const liar_batch_item* items, size_t n_items,
                                     const liar_batch_config* cfg, liar_gpu_batch** out) {
    if (!ctx || !out) return LIAR_ERR_INVALID;
    *out = nullptr;
    if (!items || n_items == 0) return ctx_fail(ctx, LIAR_ERR_INVALID, "empty batch");
    if (n_items > 65536) return ctx_fail(ctx, LIAR_ERR_INVALID, "too many items (limit 65536)");
    const int hero = cfg && cfg->hero_wavelengths ? cfg->hero_wavelengths : 1;
    if (hero != 1 && hero != 4) return ctx_fail(ctx, LIAR_ERR_INVALID, "hero_wavelengths must be 1 or 4");
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    liar_gpu_batch* b = new (std::nothrow) liar_gpu_batch();
    if (!b) return ctx_fail(ctx, LIAR_ERR_OOM, "host allocation");
    b->device = ctx->device;
    b->hero = hero;
    b->trace = (cfg && cfg->trace.block_size) ? cfg->trace : ctx->trace_cfg;
    b->shade_blocks_per_sm = (cfg && cfg->shade_blocks_per_sm) ? cfg->shade_blocks_per_sm : 16;
    if (b->shade_blocks_per_sm != 4 && b->shade_blocks_per_sm != 8 && b->shade_blocks_per_sm != 16) {
        delete b;
        return ctx_fail(ctx, LIAR_ERR_INVALID, "shade_blocks_per_sm must be 4, 8 or 16");
    }
    // unique scenes -> table; items -> path ranges
    std::vector<const liar_gpu_scene*> scenes;
    std::vector<BItem> hitems(n_items);
    std::vector<uint64_t> begin(n_items + 1, 0);
    int max_depth = 0;
    for (size_t i = 0; i < n_items; ++i) {
        const liar_batch_item& it = items[i];
        const liar_render_desc& R = it.render;
        if (!it.scene || !it.d_film || R.width <= 0 || R.height <= 0 || R.spp <= 0 || R.max_ray_generation < 0 ||
            R.tracer != LIAR_TRACER_ADJOINT_PHOTON || scene_device(it.scene) != ctx->device) {
            delete b;
            return ctx_fail(ctx, LIAR_ERR_INVALID, "batch item %zu is invalid", i);
        }
        int si = -1;
        for (size_t s = 0; s < scenes.size(); ++s)
            if (scenes[s] == it.scene) si = (int)s;
        if (si < 0) {
            si = (int)scenes.size();
            scenes.push_back(it.scene);
        }
        BItem& h = hitems[i];
        h.scene = si;
        h.width = R.width;
        h.height = R.height;
        h.spp = R.spp;
        h.max_gen = R.max_ray_generation;
        h.max_depth = R.max_depth;
        h.sampler = (uint32_t)R.sampler;
        h.seed = mix64(R.seed ^ mix64(0x51ed270b27ad0e0dull + (uint64_t)(uint32_t)R.first_sample));
        h.film = film_spec(it.d_film, R);
        if (const char* m = film_desc_error(R)) {
            delete b;
            return ctx_fail(ctx, LIAR_ERR_INVALID, "batch item %zu: %s", i, m);
        }
        h.cam = R.camera;
        h.path_begin = begin[i];
        begin[i + 1] = begin[i] + (uint64_t)R.width * R.height * R.spp;
        if ((uint64_t)R.width * R.height >= (1ull << 32)) {
            delete b;
            return ctx_fail(ctx, LIAR_ERR_INVALID, "batch item %zu: image too large", i);
        }
        if (R.max_depth <= 0) {
            delete b;
            return ctx_fail(ctx, LIAR_ERR_UNSUPPORTED, "batch item %zu: batched rendering needs max_depth > 0", i);
        }
        max_depth = std::max(max_depth, R.max_depth);
    }
    b->bounces = (cfg && cfg->max_bounces) ? cfg->max_bounces : max_depth;
    if (b->bounces < max_depth || b->bounces > 64) {
        delete b;
        return ctx_fail(ctx, LIAR_ERR_INVALID, "max_bounces must cover every item's max_depth and be <= 64");
    }
    b->total = begin[n_items];
    uint64_t W = (cfg && cfg->wave_paths > 0) ? (uint64_t)cfg->wave_paths : (1ull << 22);
    W = std::min<uint64_t>(W, std::max<uint64_t>(b->total, 1));
    W = std::min<uint64_t>(W, 1ull << 30);
    b->params.wave_paths = (uint32_t)W;
    const uint64_t waves = (b->total + W - 1) / W;
    if (waves >= (1ull << 31)) {
        delete b;
        return ctx_fail(ctx, LIAR_ERR_INVALID, "batch too large");
    }
    b->n_waves = (uint32_t)waves;
    std::vector<DScene> hs(scenes.size());
    std::vector<TreeRoot> roots(scenes.size());
    for (size_t s = 0; s < scenes.size(); ++s) {
        hs[s] = scene_dscene(scenes[s]);
        b->textured |= hs[s].n_tex > 0;
        roots[s] = TreeRoot{hs[s].nodes, hs[s].qtris};
        if (hs[s].stack_needed > (uint32_t)kTraceStackTotal) {
            delete b;
            return ctx_fail(ctx, LIAR_ERR_STACK, "a scene's tree is deeper than the trace stack");
        }
    }
    void* p = nullptr;
    rc = b_alloc(ctx, b, hs.size() * sizeof(DScene), &p, "scene table");
    if (!rc) {
        b->params.scenes = static_cast<const DScene*>(p);
        rc = ctx_cuda(ctx, cudaMemcpy(p, hs.data(), hs.size() * sizeof(DScene), cudaMemcpyHostToDevice), "scene table");
    }
    if (!rc) rc = b_alloc(ctx, b, roots.size() * sizeof(TreeRoot), &p, "tree table");
    if (!rc) {
        b->roots = static_cast<TreeRoot*>(p);
        rc = ctx_cuda(ctx, cudaMemcpy(p, roots.data(), roots.size() * sizeof(TreeRoot), cudaMemcpyHostToDevice), "tree table");
    }
    if (!rc) rc = b_alloc(ctx, b, n_items * sizeof(BItem), &p, "item table");
    if (!rc) {
        b->params.items = static_cast<const BItem*>(p);
        rc = ctx_cuda(ctx, cudaMemcpy(p, hitems.data(), n_items * sizeof(BItem), cudaMemcpyHostToDevice), "item table");
    }
    if (!rc) rc = b_alloc(ctx, b, begin.size() * 8, &p, "item ranges");
    if (!rc) {
        b->params.item_begin = static_cast<const uint64_t*>(p);
        rc = ctx_cuda(ctx, cudaMemcpy(p, begin.data(), begin.size() * 8, cudaMemcpyHostToDevice), "item ranges");
    }
    if (!rc) rc = b_alloc(ctx, b, sizeof(BControl), &p, "batch control");
    if (!rc) {
        b->ctrl = static_cast<BControl*>(p);
        b->params.ctrl = b->ctrl;
        b->params.n_items = (int)n_items;
        b->params.total_paths = b->total;
        rc = hero == 4 ? build_graph<4>(ctx, b) : build_graph<1>(ctx, b);
    }
    if (rc) {
        liar_gpu_batch_destroy(b);
        return rc;
    }
    *out = b;
    return LIAR_OK;
}

extern "C" int liar_gpu_batch_launch(liar_gpu_ctx* ctx, liar_gpu_batch* b, void* stream) {
    if (!ctx || !b) return LIAR_ERR_INVALID;
    if (b->device != ctx->device) return ctx_fail(ctx, LIAR_ERR_INVALID, "batch lives on another device");
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    return ctx_cuda(ctx, cudaGraphLaunch(b->exec, st), "batch graph launch");
}

extern "C" int liar_gpu_batch_stats(const liar_gpu_batch* b, unsigned long long* out4) {
    if (!b || !out4) return LIAR_ERR_INVALID;
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != b->device) cudaSetDevice(b->device);
    BControl c;
    const cudaError_t e = cudaMemcpy(&c, b->ctrl, sizeof(c), cudaMemcpyDeviceToHost);
    if (cur >= 0 && cur != b->device) cudaSetDevice(cur);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return LIAR_ERR_CUDA;
    }
    for (int k = 0; k < 4; ++k) out4[k] = c.stats[k];
    return LIAR_OK;
}

extern "C" void liar_gpu_batch_destroy(liar_gpu_batch* b) {
    if (!b) return;
    int cur = -1;
    cudaGetDevice(&cur);
    if (b->device >= 0) cudaSetDevice(b->device);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (void* p : b->buffers) cudaFree(p);
    if (cur >= 0) cudaSetDevice(cur);
    delete b;
}
