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
    liar_gpu_photon_map* grid[2] = {nullptr, nullptr};
    PmMaps maps;

    void release() {
        for (auto& g : grid) {
            if (g) liar_gpu_photon_map_destroy(g);
            g = nullptr;
        }
        if (mem) cudaFree(mem);
        mem = nullptr;
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
    std::vector<float> position, omega, power;
    std::vector<uint32_t> path, tag;
    uint64_t emitted = 0, stored = 0;
};

int trace(liar_gpu_ctx* ctx, const liar_gpu_scene* scene, const liar_photon_desc& pd, uint64_t capacity,
          cudaStream_t st, Traced& out) {
    for (int attempt = 0; attempt < 6; ++attempt, capacity *= 4) {
        void* mem = nullptr;
        cudaError_t e = cudaMalloc(&mem, capacity * 44 + 1024);
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
                if (e == cudaSuccess) e = cudaStreamSynchronize(st);
                if (e != cudaSuccess) rc = ctx_cuda(ctx, e, "photon download");
            }
        }
        cudaFree(mem);
        return rc;
    }
    return ctx_fail(ctx, LIAR_ERR_OOM, "photon buffer still too small");
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
    Traced T;
    int rc = trace(ctx, scene, pd, (target + pd.wave) * 4, st, T);
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
                host[6 * n + 3 * j + c] = T.power[3 * i + c] * scale;
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
