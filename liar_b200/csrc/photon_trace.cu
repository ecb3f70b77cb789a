// photon_trace.cu -- photon emission and tracing on sm_100a (the reference's PhotonMapper
// fillPhotonMaps / emitPhoton / tracePhoton, src/liar/tracers/photon_mapper.cpp:573-796).
//
// Wavefront like the path tracer: an emit kernel starts one photon per thread from a light chosen
// by power (LightContexts::sample) with SceneLight::sampleEmission(A, B) (light_point.cpp:183-190,
// light_area.cpp:256-288); the closest-hit trace kernel runs over the compacted photon queue; a
// shade kernel stores the photon at diffuse hits (one atomicAdd per stored photon into SoA
// buffers), samples the BSDF, applies the power-preserving Russian roulette
// (kernel/kernel_common.h:160-168) and appends survivors to the next queue (ballot/popc).
// Deviation: a scattered photon leaves 10 tolerances off the surface with near limit 1e-6, like
// the path tracer's rays; the reference restarts it at the hit point with near limit 0, where
// round-off can re-hit the surface it just left.
#include <cuda_runtime.h>

#include <cmath>

#include <algorithm>
#include <new>

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
int scene_device(const liar_gpu_scene* s);
}  // namespace rt
}  // namespace liar_gpu

namespace {

// photon sample dimensions (plain hashes: the photon sampler is not stratified per pixel)
enum : uint32_t {
    P_LIGHT = 0, P_A = 1, P_B = 3, P_LAMBDA = 5, P_GEN0 = 8, P_PER_GEN = 8, P_BSDF = 0, P_COMP = 2, P_RR = 3,
    P_STORE_CAUSTIC = 4, P_STORE_GLOBAL = 5
};

struct PState {
    float* lam;
    float* lam_pdf;
    float* power;
    int32_t* gen;
    uint32_t* caustic;
    uint64_t* path;
};
struct PQueue {
    liar_ray* rays;
    uint32_t* slot;
    uint32_t* count;
};
struct PParams {
    uint64_t seed;
    uint64_t first_path;
    int max_gen;
    int rt_direct;
    int final_gather;  // every diffuse hit is a global photon
    float p_global, p_caustic;  // storage probabilities (causticsQuality)
};


__device__ __forceinline__ float psample(const PParams& P, uint64_t path, uint32_t dim) {
    SampleKey k;
    k.seed = P.seed;
    k.pixel = (uint32_t)path;
    k.sample = (uint32_t)(path >> 32);
    k.spp = 1;
    return sample_dim(k, dim, false);
}

__device__ __forceinline__ void pqueue_push(const PQueue& q, bool want, const liar_ray& r, uint32_t slot) {
    const uint32_t mask = __ballot_sync(0xffffffffu, want);
    if (mask == 0) return;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(q.count, (uint32_t)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (want) {
        const uint32_t s = base + __popc(mask & ((1u << lane) - 1u));
        float4* dst = reinterpret_cast<float4*>(q.rays + s);
        dst[0] = make_float4(r.ox, r.oy, r.oz, r.tmin);
        dst[1] = make_float4(r.dx, r.dy, r.dz, r.tmax);
        q.slot[s] = slot;
    }
}

// PhotonMapper::emitPhoton for photons first_path + i
__global__ void __launch_bounds__(256) k_photon_emit(DScene S, PParams P, uint32_t n, PState st, PQueue out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool want = false;
    liar_ray r{};
    if (i < n && S.n_lights > 0) {
        const uint64_t path = P.first_path + i;
        float lpdf;
        const float lam = observer_sample(S, psample(P, path, P_LAMBDA), lpdf);
        int k = lower_bound_f(S.light_cdf, S.n_lights, psample(P, path, P_LIGHT));
        if (k > S.n_lights - 1) k = S.n_lights - 1;
        const float pc = light_choice_pdf(S, k);
        const liar_light L = S.lights[k];
        const float ax = psample(P, path, P_A), ay = psample(P, path, P_A + 1);
        const float bx = psample(P, path, P_B), by = psample(P, path, P_B + 1);
        float3 origin = mk(0, 0, 0), dir = mk(0, 0, 1);
        float pdf = 0.0f, value = 0.0f;
        if (L.type == LIAR_LIGHT_POINT) {
            // LightPoint::doSampleEmission(A, B): uniform direction from the position
            dir = uniform_sphere(ax, ay, pdf);
            origin = mk(L.pos[0], L.pos[1], L.pos[2]);
            value = spec_eval(S, L.spectrum, lam, false);
        } else if (L.type == LIAR_LIGHT_AREA_PARALLELOGRAM) {
            // LightArea::doSampleEmission(A, B): a point on the surface, a cosine-weighted direction
            const float3 u = mk(L.u[0], L.u[1], L.u[2]), v = mk(L.v[0], L.v[1], L.v[2]);
            origin = mk(L.pos[0], L.pos[1], L.pos[2]) + ax * u + ay * v;
            float3 n = normal(cross(u, v));
            const float opdf = 1.0f / S.light_area[k];
            // double-sided: the reference flips the side on 2 B.x >= 1 but then samples the
            // direction with the unmodified B (light_area.cpp:266-279)
            if (L.double_sided && 2.0f * bx >= 1.0f) n = -n;
            const float3 a = fabsf(n.x) > fabsf(n.y) ? mk(-n.z, 0.0f, n.x) : mk(0.0f, n.z, -n.y);
            const float3 tu = normal(a), tv = cross(n, tu);
            float dpdf;
            const float3 ld = cosine_hemisphere(bx, by, dpdf);
            dir = ld.x * tu + ld.y * tv + ld.z * n;
            pdf = opdf * dpdf;
            value = spec_eval(S, L.spectrum, lam, false) * ld.z;
        }
        if (pdf > 0.0f && value != 0.0f && pc > 0.0f && lpdf > 0.0f) {
            st.lam[i] = lam;
            st.lam_pdf[i] = lpdf;
            st.power[i] = value / (pc * pdf);
            st.gen[i] = 0;
            st.caustic[i] = 0;
            st.path[i] = path;
            r = liar_ray{origin.x, origin.y, origin.z, kTol, dir.x, dir.y, dir.z, INFINITY};
            want = true;
        }
    }
    pqueue_push(out, want, r, i);
}

template <bool TEX>
__global__ void __launch_bounds__(128) k_photon_shade(DScene S, PParams P, PState st, PQueue in, const liar_hit* hits,
                                                      uint32_t n_in, PQueue out, liar_photon_buffers B,
                                                      unsigned long long* counters, uint32_t* status) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    bool want = false;
    liar_ray nr{};
    uint32_t slot = 0;
    if (q < n_in) {
        slot = in.slot[q];
        const float4 r0 = reinterpret_cast<const float4*>(in.rays + q)[0];
        const float4 r1 = reinterpret_cast<const float4*>(in.rays + q)[1];
        const float3 o = mk(r0.x, r0.y, r0.z), d = mk(r1.x, r1.y, r1.z);
        const liar_hit h = hits[q];
        const int gen = st.gen[slot];
        const uint64_t path = st.path[slot];
        const float lam = st.lam[slot];
        float power = st.power[slot];
        bool caustic = st.caustic[slot] != 0;
        if (h.prim >= 0 && power != 0.0f) {
            const HitContext H = hit_context(S, o, d, (uint32_t)h.prim, h.t);
            const float3 hit_point = o + h.t * d;
            const int mi = H.mat;
            if (mi < 0) {
                // no shader: entering or leaving something, continue through
                if (gen < P.max_gen) {
                    nr = liar_ray{o.x, o.y, o.z, h.t + kTol, d.x, d.y, d.z, r1.w};
                    st.gen[slot] = gen + 1;
                    want = true;
                }
            } else if (S.mats[mi].type == LIAR_MAT_NONE) {
                // a shader without a BSDF (Unshaded) stores nothing and absorbs the photon
                // (tracePhoton: no diffuse caps, shader->bsdf() is null)
            } else {
                const liar_material M = S.mats[mi];
                if (M.type == LIAR_MAT_LAMBERT) {
                    // Shader::hasCaps(diffuse): store (photon_mapper.cpp:733-748), each map by Russian
                    // roulette with its storage probability (kept when u <= p)
                    const uint32_t sbase = P_GEN0 + P_PER_GEN * (uint32_t)gen;
                    const bool to_caustic =
                        caustic && (P.p_caustic >= 1.0f || !(psample(P, path, sbase + P_STORE_CAUSTIC) > P.p_caustic));
                    const bool to_global = (((gen > 0 || !P.rt_direct) && !caustic) || P.final_gather) &&
                                           (P.p_global >= 1.0f || !(psample(P, path, sbase + P_STORE_GLOBAL) > P.p_global));
                    if (to_caustic || to_global) {
                        const unsigned long long s = atomicAdd(counters + 0, 1ull);
                        if (s < B.capacity) {
                            const float sc = power / st.lam_pdf[slot];
                            const float3 c = observer_sensitivity(S, lam);
                            B.position[3 * s] = hit_point.x;
                            B.position[3 * s + 1] = hit_point.y;
                            B.position[3 * s + 2] = hit_point.z;
                            B.omega_in[3 * s] = -d.x;
                            B.omega_in[3 * s + 1] = -d.y;
                            B.omega_in[3 * s + 2] = -d.z;
                            B.power[3 * s] = sc * c.x;
                            B.power[3 * s + 1] = sc * c.y;
                            B.power[3 * s + 2] = sc * c.z;
                            B.path[s] = (uint32_t)path;
                            B.tag[s] = (to_caustic ? (uint32_t)LIAR_PHOTON_CAUSTIC : 0u) |
                                       (to_global ? (uint32_t)LIAR_PHOTON_GLOBAL : 0u) | ((uint32_t)gen << 8);
                            if (B.normal) {
                                B.normal[3 * s] = H.N.x;
                                B.normal[3 * s + 1] = H.N.y;
                                B.normal[3 * s + 2] = H.N.z;
                            }
                            if (to_global) atomicAdd(counters + 1, 1ull);
                            if (to_caustic) atomicAdd(counters + 2, 1ull);
                        } else {
                            atomicOr(status, 1u << 5);  // buffer full: the photon is lost, the host reports it
                        }
                    }
                }
                if (gen < P.max_gen) {
                    const Bsdf Bs = make_bsdf<TEX>(S, M, H, lam);
                    const float3 md = -d;
                    float3 wi = mk(dot(md, H.u), dot(md, H.v), dot(md, H.N));
                    wi.z = fmaxf(wi.z, kEps);
                    const uint32_t base = P_GEN0 + P_PER_GEN * (uint32_t)gen;
                    const BsdfSample smp = bsdf_sample(Bs, wi, psample(P, path, base + P_BSDF),
                                                       psample(P, path, base + P_BSDF + 1),
                                                       psample(P, path, base + P_COMP), CAP_ALL);
                    if (smp.ok()) {
                        const float cos_t = smp.wo.z;
                        float np = power * smp.value * (fabsf(cos_t) / smp.pdf);
                        const float prob = fminf(1.0f, np / power);
                        // russianRoulette(newPower, prob, u): survive when u <= prob, power / prob
                        const float u = psample(P, path, base + P_RR);
                        if (prob > 0.0f && !(u > prob)) {
                            np /= fminf(prob, 1.0f);
                            const float3 nd = smp.wo.x * H.u + smp.wo.y * H.v + smp.wo.z * H.N;
                            const float3 start = hit_point + ((cos_t > 0.0f ? 10.0f : -10.0f) * kTol) * H.ng;
                            nr = liar_ray{start.x, start.y, start.z, kTol, nd.x, nd.y, nd.z, INFINITY};
                            const bool specular = M.type != LIAR_MAT_LAMBERT;  // used caps specular or glossy
                            st.caustic[slot] = (specular && (caustic || gen == 0)) ? 1u : 0u;
                            st.power[slot] = np;
                            st.gen[slot] = gen + 1;
                            want = true;
                        }
                    }
                }
            }
        }
    }
    pqueue_push(out, want, nr, slot);
}

struct PhotonWork {
    size_t cap = 0;
    void* mem = nullptr;
    PState st{};
    PQueue q[2]{};
    liar_hit* hits = nullptr;
    unsigned long long* counters = nullptr;  // stored, global, caustic (device)
    unsigned long long* h_counters = nullptr;
    uint32_t* h_count = nullptr;
};

PhotonWork* photon_work(liar_gpu_ctx* ctx) {
    for (auto& ext : ctx->extensions)
        if (ext.first == "photon") return static_cast<PhotonWork*>(ext.second);
    PhotonWork* w = new PhotonWork();
    ctx->extensions.emplace_back("photon", w);
    ctx->on_destroy.push_back([w]() {
        if (w->mem) cudaFree(w->mem);
        if (w->counters) cudaFree(w->counters);
        if (w->h_counters) cudaFreeHost(w->h_counters);
        if (w->h_count) cudaFreeHost(w->h_count);
        delete w;
    });
    return w;
}

int ensure_photon_work(liar_gpu_ctx* ctx, PhotonWork* w, size_t n) {
    if (!w->counters) {
        cudaError_t e = cudaMalloc((void**)&w->counters, 4 * sizeof(unsigned long long));
        if (e == cudaSuccess) e = cudaMallocHost((void**)&w->h_counters, 4 * sizeof(unsigned long long));
        if (e == cudaSuccess) e = cudaMallocHost((void**)&w->h_count, 2 * sizeof(uint32_t));
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "photon counters");
    }
    if (w->cap >= n) return LIAR_OK;
    if (w->mem) cudaFree(w->mem);
    w->mem = nullptr;
    w->cap = 0;
    const size_t bytes = n * (4 * 4 + 4 + 8 + 2 * (32 + 4) + 8) + 4096;
    cudaError_t e = cudaMalloc(&w->mem, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return ctx_cuda(ctx, e, "photon wave buffers");
    }
    char* p = static_cast<char*>(w->mem);
    auto take = [&](size_t b) {
        char* r = p;
        p += (b + 255) & ~size_t(255);
        return r;
    };
    w->q[0].rays = reinterpret_cast<liar_ray*>(take(n * 32));
    w->q[1].rays = reinterpret_cast<liar_ray*>(take(n * 32));
    w->hits = reinterpret_cast<liar_hit*>(take(n * 8));
    w->st.path = reinterpret_cast<uint64_t*>(take(n * 8));
    w->q[0].slot = reinterpret_cast<uint32_t*>(take(n * 4));
    w->q[1].slot = reinterpret_cast<uint32_t*>(take(n * 4));
    w->st.lam = reinterpret_cast<float*>(take(n * 4));
    w->st.lam_pdf = reinterpret_cast<float*>(take(n * 4));
    w->st.power = reinterpret_cast<float*>(take(n * 4));
    w->st.gen = reinterpret_cast<int32_t*>(take(n * 4));
    w->st.caustic = reinterpret_cast<uint32_t*>(take(n * 4));
    w->q[0].count = reinterpret_cast<uint32_t*>(take(4));
    w->q[1].count = reinterpret_cast<uint32_t*>(take(4));
    w->cap = n;
    return LIAR_OK;
}

}  // namespace

extern "C" int liar_gpu_photon_trace(liar_gpu_ctx* ctx, const liar_gpu_scene* scene, const liar_photon_desc* desc,
                                     const liar_photon_buffers* out, liar_photon_counts* counts, void* stream) {
    if (!ctx) return LIAR_ERR_INVALID;
    if (!scene || !desc || !out || !counts) return ctx_fail(ctx, LIAR_ERR_INVALID, "null scene, description or buffers");
    if (scene_device(scene) != ctx->device) return ctx_fail(ctx, LIAR_ERR_INVALID, "scene lives on another device");
    if (!out->position || !out->omega_in || !out->power || !out->path || !out->tag || out->capacity == 0)
        return ctx_fail(ctx, LIAR_ERR_INVALID, "photon buffers incomplete");
    if (desc->max_ray_generation < 0) return ctx_fail(ctx, LIAR_ERR_INVALID, "max_ray_generation must be >= 0");
    if (desc->max_emitted >= (1ull << 32)) return ctx_fail(ctx, LIAR_ERR_INVALID, "max_emitted must be < 2^32");
    // photons leave point lights and parallelogram area lights; other lights are never chosen for
    // emission successfully (their emission pdf is zero here), which the counts show as emitted
    // photons that stored nothing
    const DScene& S = scene_dscene(scene);
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    PhotonWork* w = photon_work(ctx);
    uint64_t wave = desc->wave ? desc->wave : (1ull << 21);
    wave = std::min<uint64_t>(wave, std::max<uint64_t>(desc->max_emitted, 1));
    rc = ensure_photon_work(ctx, w, (size_t)wave);
    if (rc) return rc;
    cudaError_t e = cudaMemsetAsync(w->counters, 0, 4 * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "photon counters");
    PParams P;
    P.seed = mix64(desc->seed ^ 0x9a1d37c8e15b22f3ull);
    P.max_gen = desc->max_ray_generation;
    P.rt_direct = desc->ray_traced_direct;
    P.final_gather = desc->final_gather ? 1 : 0;
    if (!std::isfinite(desc->caustics_quality)) return ctx_fail(ctx, LIAR_ERR_INVALID, "caustics quality is not finite");
    storage_probabilities(desc->caustics_quality, P.p_global, P.p_caustic);
    uint64_t emitted = 0;
    counts->stored = counts->global = counts->caustic = 0;
    while (emitted < desc->max_emitted && counts->global < desc->global_target) {
        const uint32_t n = (uint32_t)std::min<uint64_t>(wave, desc->max_emitted - emitted);
        P.first_path = emitted;
        int cur = 0;
        e = cudaMemsetAsync(w->q[0].count, 0, 4, st);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "photon queue");
        k_photon_emit<<<(n + 255) / 256, 256, 0, st>>>(S, P, n, w->st, w->q[0]);
        e = cudaMemcpyAsync(w->h_count, w->q[0].count, 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "photon emit");
        uint32_t n_in = w->h_count[0];
        for (int bounce = 0; n_in > 0; ++bounce) {
            if (bounce > desc->max_ray_generation + 2) break;
            rc = trace_mesh_internal(ctx, scene_mesh(scene), w->q[cur].rays, n_in, w->hits, 0, st, kCounterWord + 9);
            if (rc) return rc;
            e = cudaMemsetAsync(w->q[cur ^ 1].count, 0, 4, st);
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "photon queue");
            (S.n_tex > 0 ? k_photon_shade<true> : k_photon_shade<false>)<<<(n_in + 127) / 128, 128, 0, st>>>(S, P, w->st, w->q[cur], w->hits, n_in, w->q[cur ^ 1], *out,
                                                               w->counters, ctx->d_scratch + kStatusWord);
            cur ^= 1;
            e = cudaMemcpyAsync(w->h_count, w->q[cur].count, 4, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "photon shade");
            n_in = w->h_count[0];
        }
        e = cudaMemcpyAsync(w->h_counters, w->counters, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "photon counters");
        emitted += n;
        counts->stored = w->h_counters[0];
        counts->global = w->h_counters[1];
        counts->caustic = w->h_counters[2];
        if (counts->stored > out->capacity) {
            counts->emitted = emitted;
            counts->stored = out->capacity;
            ctx_check_status(ctx);  // clears the device's buffer-full bit
            return ctx_fail(ctx, LIAR_ERR_OOM, "photon buffer full after %llu emitted photons",
                            (unsigned long long)emitted);
        }
    }
    counts->emitted = emitted;
    return ctx_check_status(ctx);
}
