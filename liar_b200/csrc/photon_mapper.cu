// photon_mapper.cu -- the PhotonMapper tracer (src/liar/tracers/photon_mapper.cpp) on sm_100a:
// the photon maps of a render, then the DirectLighting wavefront (direct.cu) with the maps'
// estimates at every vertex that has a diffuse part.
//
// Maps (PhotonMapper::doPreProcess, :372-390): photons are traced on the GPU by
// liar_gpu_photon_trace (photon_trace.cu: fillPhotonMaps / emitPhoton / tracePhoton) in waves;
// the reference stops emitting as soon as the global map holds globalMapSize photons, so the
// photons of emissions after the one that filled it are dropped and "photons shot" is that
// emission's index + 1. Photons are put in the reference's buffer order (emission, then bounce),
// their XYZ power scaled by 1 / photons shot (buildPhotonMap, :798-813), the automatic estimation
// radius is sqrt(size x power of the middle photon of the buffer / tolerance) / pi (:815-833, the
// middle of the unsorted buffer, as there), every power gets its spectral blend (the standard
// recovery, Spectral::fromXYZ), and a gather grid is built over each map (photon.cu).
// The maps are kept for the next render of the same scene and settings.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/liar_gpu.h"
#include "ctx.h"
#include "photon_mapper.h"
#include "sampler.h"

using namespace liar_gpu;

namespace liar_gpu {
namespace rt {
uint64_t scene_uid(const liar_gpu_scene* s);
}  // namespace rt
const DRecovery* ctx_recovery(liar_gpu_ctx* ctx);
int recovery_locate_device(liar_gpu_ctx* ctx, const float* d_xyz, size_t n, int32_t* d_idx, float* d_w,
                           cudaStream_t st);
}  // namespace liar_gpu

namespace {

struct PmCache {
    uint64_t scene = 0;
    liar_photon_mapper_desc desc{};
    int max_gen = -1;
    uint64_t seed = 0;
    bool valid = false;
    void* mem = nullptr;
    void* irr_mem = nullptr;
    liar_gpu_photon_map* grid[2] = {nullptr, nullptr};
    liar_gpu_photon_map* irr_grid = nullptr;
    PmMaps maps;

    void release() {
        for (auto& g : grid) {
            if (g) liar_gpu_photon_map_destroy(g);
            g = nullptr;
        }
        if (irr_grid) liar_gpu_photon_map_destroy(irr_grid);
        irr_grid = nullptr;
        if (mem) cudaFree(mem);
        if (irr_mem) cudaFree(irr_mem);
        mem = irr_mem = nullptr;
        valid = false;
    }
};

PmCache* pm_cache(liar_gpu_ctx* ctx) {
    for (auto& ext : ctx->extensions)
        if (ext.first == "photon_mapper") return static_cast<PmCache*>(ext.second);
    PmCache* c = new PmCache();
    ctx->extensions.emplace_back("photon_mapper", c);
    ctx->on_destroy.push_back([c]() {
        c->release();
        delete c;
    });
    return c;
}

bool same_desc(const liar_photon_mapper_desc& a, const liar_photon_mapper_desc& b) {
    return std::memcmp(&a, &b, sizeof(a)) == 0;
}

// the stored photons of one trace, on the host
struct Traced {
    std::vector<float> position, omega, power, normal;
    std::vector<uint32_t> path, tag;
    uint64_t emitted = 0, stored = 0;
};

int trace(liar_gpu_ctx* ctx, const liar_gpu_scene* scene, const liar_photon_desc& pd, uint64_t capacity,
          cudaStream_t st, Traced& out) {
    for (int attempt = 0; attempt < 6; ++attempt, capacity *= 4) {
        void* mem = nullptr;
        cudaError_t e = cudaMalloc(&mem, capacity * 56 + 1024);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return ctx_cuda(ctx, e, "photon buffers");
        }
        char* p = static_cast<char*>(mem);
        liar_photon_buffers B;
        B.position = reinterpret_cast<float*>(p);
        B.omega_in = reinterpret_cast<float*>(p + capacity * 12);
        B.power = reinterpret_cast<float*>(p + capacity * 24);
        B.path = reinterpret_cast<uint32_t*>(p + capacity * 36);
        B.tag = reinterpret_cast<uint32_t*>(p + capacity * 40);
        B.normal = reinterpret_cast<float*>(p + capacity * 44);
        B.capacity = capacity;
        liar_photon_counts counts{};
        int rc = liar_gpu_photon_trace(ctx, scene, &pd, &B, &counts, st);
        if (rc == LIAR_ERR_OOM) {
            cudaFree(mem);
            continue;  // more photons than the buffer holds: the same photons again into a larger one
        }
        if (rc == LIAR_OK) {
            const size_t n = (size_t)counts.stored;
            out.position.resize(3 * n);
            out.omega.resize(3 * n);
            out.power.resize(3 * n);
            out.normal.resize(3 * n);
            out.path.resize(n);
            out.tag.resize(n);
            out.emitted = counts.emitted;
            out.stored = n;
            if (n) {
                e = cudaMemcpyAsync(out.position.data(), B.position, n * 12, cudaMemcpyDeviceToHost, st);
                if (e == cudaSuccess) e = cudaMemcpyAsync(out.omega.data(), B.omega_in, n * 12, cudaMemcpyDeviceToHost, st);
                if (e == cudaSuccess) e = cudaMemcpyAsync(out.power.data(), B.power, n * 12, cudaMemcpyDeviceToHost, st);
                if (e == cudaSuccess) e = cudaMemcpyAsync(out.path.data(), B.path, n * 4, cudaMemcpyDeviceToHost, st);
                if (e == cudaSuccess) e = cudaMemcpyAsync(out.tag.data(), B.tag, n * 4, cudaMemcpyDeviceToHost, st);
                if (e == cudaSuccess) e = cudaMemcpyAsync(out.normal.data(), B.normal, n * 12, cudaMemcpyDeviceToHost, st);
                if (e == cudaSuccess) e = cudaStreamSynchronize(st);
                if (e != cudaSuccess) rc = ctx_cuda(ctx, e, "photon download");
            }
        }
        cudaFree(mem);
        return rc;
    }
    return ctx_fail(ctx, LIAR_ERR_OOM, "photon buffer still too small");
}

__global__ void k_irr_r2(const float* __restrict__ d2, const int32_t* __restrict__ cnt, uint32_t n, int k,
                         float* __restrict__ r2) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = min(cnt[i], k);
    r2[i] = c > 0 ? d2[(size_t)i * k + c - 1] : 0.0f;
}

// the points of the irradiance map: global photons chosen with probability `ratio` (the reference
// draws uniform(rng) <= ratio per stored global photon; here a hash of the photon's emission and
// bounce), each with the photon's position and normal; their irradiance is estimateIrradianceImpl
// over the global map (liar_gpu_photon_estimate_device), and a gather grid over them answers the
// nearest-neighbour queries of estimateRadiance
int build_irradiance(liar_gpu_ctx* ctx, cudaStream_t st, PmCache* C, const Traced& T,
                     const std::vector<uint32_t>& global, float ratio) {
    PmMaps& M = C->maps;
    const PmMap& G = M.map[kPmGlobal];
    std::vector<float> host;  // positions, then normals
    std::vector<uint32_t> chosen;
    for (uint32_t i : global) {
        const uint64_t h = mix64(0x6972726164ull ^ mix64(((uint64_t)T.path[i] << 8) | ((T.tag[i] >> 8) & 0xffu)));
        const float u = (float)(h >> 40) * (1.0f / 16777216.0f);
        if (u <= ratio) chosen.push_back(i);
    }
    const size_t n = chosen.size();
    if (n == 0) return LIAR_OK;
    host.resize(6 * n);
    for (size_t j = 0; j < n; ++j)
        for (int c = 0; c < 3; ++c) {
            host[3 * j + c] = T.position[3 * chosen[j] + c];
            host[3 * n + 3 * j + c] = T.normal[3 * chosen[j] + c];
        }
    const int k = G.k;
    // per point: position, normal, xyz, blend (idx, w) = 60 B and r2 4 B; gather scratch k x 8 B + 4 B
    const size_t keep = n * 64 + 1024, scratch = n * ((size_t)k * 8 + 4) + 256;
    cudaError_t e = cudaMalloc(&C->irr_mem, keep);
    void* tmp = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&tmp, scratch);
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (tmp) cudaFree(tmp);
        return ctx_cuda(ctx, e, "irradiance map");
    }
    float* pos = static_cast<float*>(C->irr_mem);
    float* nrm = pos + 3 * n;
    float* xyz = pos + 6 * n;
    int32_t* bidx = reinterpret_cast<int32_t*>(pos + 9 * n);
    float* bw = pos + 12 * n;
    float* r2 = pos + 15 * n;
    int32_t* g_idx = static_cast<int32_t*>(tmp);
    float* g_d2 = reinterpret_cast<float*>(g_idx + (size_t)n * k);
    int32_t* g_cnt = reinterpret_cast<int32_t*>(g_d2 + (size_t)n * k);
    int rc = LIAR_OK;
    e = cudaMemcpyAsync(pos, host.data(), 6 * n * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) rc = ctx_cuda(ctx, e, "irradiance points");
    if (!rc) rc = liar_gpu_photon_gather_device(ctx, G.grid, pos, n, k, g_idx, g_d2, g_cnt, st);
    if (!rc)
        rc = liar_gpu_photon_estimate_device(ctx, G.power, G.omega_in, (size_t)G.n, nrm, n, k, g_idx, g_d2, g_cnt, 1.0f,
                                             xyz, st);
    if (!rc) {
        k_irr_r2<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g_d2, g_cnt, (uint32_t)n, k, r2);
        rc = ctx_cuda(ctx, cudaGetLastError(), "irradiance radii");
    }
    if (!rc) rc = recovery_locate_device(ctx, xyz, n, bidx, bw, st);
    if (!rc) rc = liar_gpu_photon_map_build_device(ctx, pos, n, G.radius, &C->irr_grid, st);
    e = cudaStreamSynchronize(st);
    cudaFree(tmp);
    if (rc) return rc;
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "irradiance map");
    PmIrradiance& I = M.irr;
    I.grid = C->irr_grid;
    I.position = pos;
    I.normal = nrm;
    I.xyz = xyz;
    I.blend_idx = bidx;
    I.blend_w = bw;
    I.r2 = r2;
    I.n = n;
    return LIAR_OK;
}

int build_maps(liar_gpu_ctx* ctx, const liar_gpu_scene* scene, const liar_render_desc& R, cudaStream_t st,
               PmCache* C) {
    const liar_photon_mapper_desc& D = R.photon_mapper;
    const uint64_t max_photons = D.max_photons ? D.max_photons : 100000000ull;
    const uint64_t target = D.global_map_size ? D.global_map_size : 10000ull;
    liar_photon_desc pd{};
    pd.max_ray_generation = R.max_ray_generation;
    pd.ray_traced_direct = D.ray_trace_direct < 0 ? 0 : 1;
    pd.seed = R.seed ^ 0x70686f746f6e73ull;
    pd.global_target = target;
    pd.max_emitted = max_photons;
    pd.wave = std::min<uint64_t>(std::max<uint64_t>(2 * target, 1u << 14), 1u << 21);
    const bool fg = D.ray_trace_direct >= 0 && D.final_gather_rays > 0;  // hasFinalGather
    pd.final_gather = fg ? 1 : 0;
    pd.caustics_quality = D.caustics_quality;
    float p_store[2];  // storage probabilities of the global and caustic maps
    storage_probabilities(D.caustics_quality, p_store[kPmGlobal], p_store[kPmCaustic]);
    // a global map filled at probability p takes about 1 / p more emissions (and their caustics)
    const uint64_t more = (uint64_t)std::ceil(1.0 / std::max(p_store[kPmGlobal], 1e-6f));
    Traced T;
    int rc = trace(ctx, scene, pd, (target * more + pd.wave) * 4, st, T);
    if (rc) return rc;
    // the reference's buffer order: by emission, then by bounce (the generation is in tag >> 8)
    std::vector<uint32_t> order(T.stored);
    for (uint32_t i = 0; i < order.size(); ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        return T.path[a] != T.path[b] ? T.path[a] < T.path[b] : (T.tag[a] >> 8) < (T.tag[b] >> 8);
    });
    // fillPhotonMaps stops after the emission that brought the global map to `target` photons
    uint64_t shot = T.emitted, n_global = 0;
    for (uint32_t i : order)
        if ((T.tag[i] & LIAR_PHOTON_GLOBAL) && ++n_global == target) {
            shot = (uint64_t)T.path[i] + 1;
            break;
        }
    if (shot == 0) return ctx_fail(ctx, LIAR_ERR_INVALID, "no photons were emitted");
    const float scale = 1.0f / (float)shot;  // powerScale = num::inv(photonsShot)
    C->release();
    PmMaps& M = C->maps;
    M = PmMaps();
    M.emitted = shot;
    M.visualize = D.visualize != 0;
    M.ray_direct = D.ray_trace_direct < 0 ? 0 : 1;
    M.fg_rays = fg ? D.final_gather_rays : 0;
    M.fg_secondary = fg ? (D.secondary_gather_rays == 0 ? 1 : std::max(0, D.secondary_gather_rays)) : 0;
    std::vector<uint32_t> members[2];
    for (uint32_t i : order)
        if (T.path[i] < shot) {
            if (T.tag[i] & LIAR_PHOTON_GLOBAL) members[kPmGlobal].push_back(i);
            if (T.tag[i] & LIAR_PHOTON_CAUSTIC) members[kPmCaustic].push_back(i);
        }
    // one allocation: per map position, omega, power (3 floats each), blend indices and weights
    size_t total = 0;
    for (int m = 0; m < 2; ++m) total += ((members[m].size() * 60 + 255) & ~size_t(255)) + 256;
    cudaError_t e = cudaMalloc(&C->mem, std::max<size_t>(total, 256));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return ctx_cuda(ctx, e, "photon maps");
    }
    char* base = static_cast<char*>(C->mem);
    const DRecovery* rec = ctx_recovery(ctx);
    M.rec = *rec;
    for (int m = 0; m < 2; ++m) {
        const size_t n = members[m].size();
        PmMap& P = M.map[m];
        const int k = D.estimation_size[m] > 0 ? D.estimation_size[m] : 50;
        P.k = k;
        P.n = n;
        std::vector<float> host(9 * n);
        for (size_t j = 0; j < n; ++j) {
            const uint32_t i = members[m][j];
            for (int c = 0; c < 3; ++c) {
                host[3 * j + c] = T.position[3 * i + c];
                host[3 * n + 3 * j + c] = T.omega[3 * i + c];
                host[6 * n + 3 * j + c] = T.power[3 * i + c] * (scale / p_store[m]);  // russianRoulette's power / p
            }
        }
        float radius = D.estimation_radius[m];
        if (radius == 0.0f && n > 0) {
            const float tol = D.estimation_tolerance[m] > 0.0f ? D.estimation_tolerance[m] : 0.05f;
            const size_t mid = n / 2;
            const float median = std::fabs(host[6 * n + 3 * mid]) + std::fabs(host[6 * n + 3 * mid + 1]) +
                                 std::fabs(host[6 * n + 3 * mid + 2]);
            const float area = (float)k * median / tol;
            radius = std::sqrt(area) / 3.14159265358979323846f;
        }
        P.radius = radius;
        float* dpos = reinterpret_cast<float*>(base);
        P.position = dpos;
        P.omega_in = dpos + 3 * n;
        P.power = dpos + 6 * n;
        int32_t* didx = reinterpret_cast<int32_t*>(dpos + 9 * n);
        float* dw = reinterpret_cast<float*>(didx + 3 * n);
        P.blend_idx = didx;
        P.blend_w = dw;
        base += ((n * 60 + 255) & ~size_t(255)) + 256;
        if (n == 0) continue;
        e = cudaMemcpyAsync(dpos, host.data(), 9 * n * sizeof(float), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "photon map upload");
        rc = recovery_locate_device(ctx, P.power, n, didx, dw, st);
        if (rc) return rc;
        if (!(radius > 0.0f)) return ctx_fail(ctx, LIAR_ERR_INVALID, "photon map %d: estimation radius not positive", m);
        rc = liar_gpu_photon_map_build_device(ctx, dpos, n, radius, &C->grid[m], st);
        if (rc) return rc;
        P.grid = C->grid[m];
        e = cudaStreamSynchronize(st);  // the host copy of the photons goes out of scope
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "photon map build");
    }
    // ---- the irradiance map of final gathering (photon_mapper.cpp:745-749, 970-995)
    const float ratio = D.ratio_precomputed_irradiance == 0.0f ? 0.25f : D.ratio_precomputed_irradiance;
    if (fg && ratio > 0.0f && M.map[kPmGlobal].n > 0) {
        rc = build_irradiance(ctx, st, C, T, members[kPmGlobal], ratio);
        if (rc) return rc;
    }
    C->scene = rt::scene_uid(scene);
    C->desc = D;
    C->max_gen = R.max_ray_generation;
    C->seed = R.seed;
    C->valid = true;
    return LIAR_OK;
}

}  // namespace

namespace liar_gpu {
namespace rt {

int render_photon_mapper(liar_gpu_ctx* ctx, const liar_gpu_scene* scene, const liar_render_desc& R, float* d_film,
                         cudaStream_t st) {
    const liar_photon_mapper_desc& D = R.photon_mapper;
    for (int m = 0; m < 2; ++m) {
        if (D.estimation_size[m] < 0 || D.estimation_size[m] > 64)
            return ctx_fail(ctx, LIAR_ERR_UNSUPPORTED, "photon map %d: estimation size must be 1..64 (0 = 50)", m);
        if (!(D.estimation_radius[m] >= 0.0f) || !(D.estimation_tolerance[m] >= 0.0f))
            return ctx_fail(ctx, LIAR_ERR_INVALID, "photon map %d: negative estimation radius or tolerance", m);
    }
    if (D.max_photons >= (1ull << 32)) return ctx_fail(ctx, LIAR_ERR_INVALID, "max_photons must be < 2^32");
    if (!ctx_recovery(ctx))
        return ctx_fail(ctx, LIAR_ERR_INVALID, "the PhotonMapper needs the context's recovery table (liar_gpu_set_recovery)");
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    PmCache* C = pm_cache(ctx);
    if (!(C->valid && C->scene == scene_uid(scene) && same_desc(C->desc, D) && C->max_gen == R.max_ray_generation &&
          C->seed == R.seed)) {
        rc = build_maps(ctx, scene, R, st, C);
        if (rc) {
            C->release();
            return rc;
        }
    }
    return render_direct(ctx, scene, R, d_film, st, &C->maps);
}

}  // namespace rt
}  // namespace liar_gpu

extern "C" int liar_gpu_photon_mapper_stats(const liar_gpu_ctx* ctx, unsigned long long* out4, float* radii) {
    if (!ctx || !out4) return LIAR_ERR_INVALID;
    for (int k = 0; k < 4; ++k) out4[k] = 0;
    for (auto& ext : ctx->extensions)
        if (ext.first == "photon_mapper") {
            const PmCache* c = static_cast<const PmCache*>(ext.second);
            if (!c->valid) break;
            out4[0] = c->maps.emitted;
            out4[1] = c->maps.map[kPmGlobal].n;
            out4[2] = c->maps.map[kPmCaustic].n;
            out4[3] = 1;
            if (radii) {
                radii[0] = c->maps.map[kPmGlobal].radius;
                radii[1] = c->maps.map[kPmCaustic].radius;
            }
        }
    return LIAR_OK;
}

extern "C" int liar_gpu_photon_mapper_get_map(liar_gpu_ctx* ctx, int map, float* position, float* omega_in,
                                              float* power, int32_t* blend_idx, float* blend_w, size_t capacity,
                                              size_t* n_out) {
    if (!ctx || !n_out) return LIAR_ERR_INVALID;
    if (map != kPmGlobal && map != kPmCaustic) return ctx_fail(ctx, LIAR_ERR_INVALID, "map must be 0 (global) or 1 (caustic)");
    *n_out = 0;
    const PmCache* c = nullptr;
    for (auto& ext : ctx->extensions)
        if (ext.first == "photon_mapper") c = static_cast<const PmCache*>(ext.second);
    if (!c || !c->valid) return ctx_fail(ctx, LIAR_ERR_INVALID, "no photon maps on this context");
    const PmMap& M = c->maps.map[map];
    *n_out = (size_t)M.n;
    if (M.n > capacity) return ctx_fail(ctx, LIAR_ERR_INVALID, "map holds %llu photons, more than capacity",
                                        (unsigned long long)M.n);
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    cudaError_t e = cudaSuccess;
    const size_t n = (size_t)M.n;
    if (n && position) e = cudaMemcpy(position, M.position, n * 12, cudaMemcpyDeviceToHost);
    if (n && e == cudaSuccess && omega_in) e = cudaMemcpy(omega_in, M.omega_in, n * 12, cudaMemcpyDeviceToHost);
    if (n && e == cudaSuccess && power) e = cudaMemcpy(power, M.power, n * 12, cudaMemcpyDeviceToHost);
    if (n && e == cudaSuccess && blend_idx) e = cudaMemcpy(blend_idx, M.blend_idx, n * 12, cudaMemcpyDeviceToHost);
    if (n && e == cudaSuccess && blend_w) e = cudaMemcpy(blend_w, M.blend_w, n * 12, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? LIAR_OK : ctx_cuda(ctx, e, "photon map download");
}

extern "C" int liar_gpu_photon_mapper_get_irradiance(liar_gpu_ctx* ctx, float* position, float* normal, float* xyz,
                                                     int32_t* blend_idx, float* blend_w, float* r2, size_t capacity,
                                                     size_t* n_out) {
    if (!ctx || !n_out) return LIAR_ERR_INVALID;
    *n_out = 0;
    const PmCache* c = nullptr;
    for (auto& ext : ctx->extensions)
        if (ext.first == "photon_mapper") c = static_cast<const PmCache*>(ext.second);
    if (!c || !c->valid) return ctx_fail(ctx, LIAR_ERR_INVALID, "no photon maps on this context");
    const PmIrradiance& I = c->maps.irr;
    *n_out = (size_t)I.n;
    if (I.n > capacity) return ctx_fail(ctx, LIAR_ERR_INVALID, "irradiance map holds %llu points, more than capacity",
                                        (unsigned long long)I.n);
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    const size_t n = (size_t)I.n;
    cudaError_t e = cudaSuccess;
    const void* src[6] = {I.position, I.normal, I.xyz, I.blend_idx, I.blend_w, I.r2};
    void* dst[6] = {position, normal, xyz, blend_idx, blend_w, r2};
    const size_t bytes[6] = {n * 12, n * 12, n * 12, n * 12, n * 12, n * 4};
    for (int k = 0; k < 6 && e == cudaSuccess; ++k)
        if (n && dst[k]) e = cudaMemcpy(dst[k], src[k], bytes[k], cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? LIAR_OK : ctx_cuda(ctx, e, "irradiance map download");
}
