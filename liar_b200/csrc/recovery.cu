// recovery.cu -- the standard tristimulus-to-spectrum recovery table of a context
// (liar_gpu_set_recovery, the reference's liar.Recovery.setStandard with a RecoveryMengSimon,
// src/liar/__init__.py:72-79) and the location of colours in it on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/liar_gpu.h"
#include "ctx.h"
#include "recovery.cuh"

using namespace liar_gpu;

namespace {

struct RecoveryTable {
    void* mem = nullptr;
    DRecovery d{};
    bool set = false;
    std::vector<void*> retired;  // replaced tables, still read by the scenes and maps built with them
};

RecoveryTable* recovery_table(liar_gpu_ctx* ctx) {
    for (auto& ext : ctx->extensions)
        if (ext.first == "recovery") return static_cast<RecoveryTable*>(ext.second);
    RecoveryTable* t = new RecoveryTable();
    ctx->extensions.emplace_back("recovery", t);
    ctx->on_destroy.push_back([t]() {
        if (t->mem) cudaFree(t->mem);
        for (void* p : t->retired) cudaFree(p);
        delete t;
    });
    return t;
}

constexpr int kGrid = 64;

__global__ void k_recovery_locate(DRecovery R, const float* __restrict__ xyz, size_t n, int32_t* __restrict__ idx,
                                  float* __restrict__ w) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        RecoveryBlend b;
        if (!recovery_locate(R, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], b)) {
            b.idx[0] = b.idx[1] = b.idx[2] = -1;
            b.w[0] = b.w[1] = b.w[2] = 0.0f;
        }
        for (int j = 0; j < 3; ++j) {
            idx[3 * i + j] = b.idx[j];
            w[3 * i + j] = b.w[j];
        }
    }
}

}  // namespace

namespace liar_gpu {
// the context's recovery table, or nullptr when none was set
const DRecovery* ctx_recovery(liar_gpu_ctx* ctx) {
    for (auto& ext : ctx->extensions)
        if (ext.first == "recovery") {
            RecoveryTable* t = static_cast<RecoveryTable*>(ext.second);
            return t->set ? &t->d : nullptr;
        }
    return nullptr;
}

int recovery_locate_device(liar_gpu_ctx* ctx, const float* d_xyz, size_t n, int32_t* d_idx, float* d_w,
                           cudaStream_t st) {
    const DRecovery* R = ctx_recovery(ctx);
    if (!R) return ctx_fail(ctx, LIAR_ERR_INVALID, "no recovery table set on this context (liar_gpu_set_recovery)");
    if (n == 0) return LIAR_OK;
    const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)ctx->num_sms * 8);
    k_recovery_locate<<<blocks, 256, 0, st>>>(*R, d_xyz, n, d_idx, d_w);
    return ctx_cuda(ctx, cudaGetLastError(), "recovery location");
}
}  // namespace liar_gpu

extern "C" int liar_gpu_set_recovery(liar_gpu_ctx* ctx, const float* wavelengths, int n_wavelengths, const float* xy,
                                     const float* spectra, int n_samples, const int32_t* triangles, int n_triangles) {
    if (!ctx) return LIAR_ERR_INVALID;
    if (!wavelengths || !xy || !spectra || !triangles || n_wavelengths < 2 || n_samples < 1 || n_triangles < 1)
        return ctx_fail(ctx, LIAR_ERR_INVALID, "recovery table: null arrays or empty table");
    for (int k = 1; k < n_wavelengths; ++k)
        if (!(wavelengths[k] > wavelengths[k - 1]))
            return ctx_fail(ctx, LIAR_ERR_INVALID, "recovery table: wavelengths must increase strictly");
    std::vector<float> pts(2 * (size_t)(n_samples + 4));
    for (int i = 0; i < n_samples; ++i) {
        const float x = xy[2 * i], y = xy[2 * i + 1];
        if (!(x >= kRecoveryBoxLoX && x <= kRecoveryBoxHiX && y >= kRecoveryBoxLoY && y <= kRecoveryBoxHiY))
            return ctx_fail(ctx, LIAR_ERR_INVALID, "recovery table: chromaticity %d outside the box", i);
        pts[2 * i] = x;
        pts[2 * i + 1] = y;
    }
    const float corners[8] = {kRecoveryBoxLoX, kRecoveryBoxLoY, kRecoveryBoxHiX, kRecoveryBoxLoY,
                              kRecoveryBoxHiX, kRecoveryBoxHiY, kRecoveryBoxLoX, kRecoveryBoxHiY};
    for (int c = 0; c < 8; ++c) pts[2 * (size_t)n_samples + c] = corners[c];
    for (int t = 0; t < 3 * n_triangles; ++t)
        if (triangles[t] < 0 || triangles[t] >= n_samples + 4)
            return ctx_fail(ctx, LIAR_ERR_INVALID, "recovery table: triangle corner out of range");
    std::vector<float> maxima(n_samples);
    for (int i = 0; i < n_samples; ++i) {
        float m = -INFINITY;
        for (int k = 0; k < n_wavelengths; ++k) m = std::max(m, spectra[(size_t)i * n_wavelengths + k]);
        maxima[i] = m;  // PointInfo::max
    }
    // the grid: every triangle in the cells its bounding box meets
    const float cw = (kRecoveryBoxHiX - kRecoveryBoxLoX) / kGrid, ch = (kRecoveryBoxHiY - kRecoveryBoxLoY) / kGrid;
    std::vector<std::vector<int32_t>> cells((size_t)kGrid * kGrid);
    for (int t = 0; t < n_triangles; ++t) {
        float x0 = INFINITY, y0 = INFINITY, x1 = -INFINITY, y1 = -INFINITY;
        for (int j = 0; j < 3; ++j) {
            const int i = triangles[3 * t + j];
            x0 = std::min(x0, pts[2 * i]);
            x1 = std::max(x1, pts[2 * i]);
            y0 = std::min(y0, pts[2 * i + 1]);
            y1 = std::max(y1, pts[2 * i + 1]);
        }
        const int cx0 = std::max(0, (int)std::floor((x0 - kRecoveryBoxLoX) / cw) - 1);
        const int cx1 = std::min(kGrid - 1, (int)std::floor((x1 - kRecoveryBoxLoX) / cw) + 1);
        const int cy0 = std::max(0, (int)std::floor((y0 - kRecoveryBoxLoY) / ch) - 1);
        const int cy1 = std::min(kGrid - 1, (int)std::floor((y1 - kRecoveryBoxLoY) / ch) + 1);
        for (int cy = cy0; cy <= cy1; ++cy)
            for (int cx = cx0; cx <= cx1; ++cx) cells[(size_t)cy * kGrid + cx].push_back(t);
    }
    std::vector<int32_t> first(1, 0), flat;
    for (const auto& c : cells) {
        flat.insert(flat.end(), c.begin(), c.end());
        first.push_back((int32_t)flat.size());
    }
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    RecoveryTable* T = recovery_table(ctx);
    if (T->mem) {
        T->retired.push_back(T->mem);
        T->mem = nullptr;
        T->set = false;
    }
    const size_t nw = (size_t)n_wavelengths, ns = (size_t)n_samples;
    const size_t sizes[7] = {nw * 4, ns * nw * 4, ns * 4, pts.size() * 4, (size_t)n_triangles * 12, first.size() * 4,
                             std::max<size_t>(flat.size(), 1) * 4};
    size_t total = 0;
    for (size_t b : sizes) total += (b + 255) & ~size_t(255);
    cudaError_t e = cudaMalloc(&T->mem, total);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return ctx_cuda(ctx, e, "recovery table");
    }
    char* p = static_cast<char*>(T->mem);
    void* dst[7];
    for (int k = 0; k < 7; ++k) {
        dst[k] = p;
        p += (sizes[k] + 255) & ~size_t(255);
    }
    const void* src[7] = {wavelengths, spectra, maxima.data(), pts.data(), triangles, first.data(), flat.data()};
    for (int k = 0; k < 7 && e == cudaSuccess; ++k)
        if (k < 6 || !flat.empty()) e = cudaMemcpy(dst[k], src[k], sizes[k], cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "recovery table upload");
    DRecovery& d = T->d;
    d.wavelengths = static_cast<const float*>(dst[0]);
    d.spectra = static_cast<const float*>(dst[1]);
    d.maxima = static_cast<const float*>(dst[2]);
    d.points = static_cast<const float*>(dst[3]);
    d.tris = static_cast<const int32_t*>(dst[4]);
    d.cell_first = static_cast<const int32_t*>(dst[5]);
    d.cell_tris = static_cast<const int32_t*>(dst[6]);
    d.n_w = n_wavelengths;
    d.n_s = n_samples;
    d.n_t = n_triangles;
    d.gx = d.gy = kGrid;
    d.lo_x = kRecoveryBoxLoX;
    d.lo_y = kRecoveryBoxLoY;
    d.inv_cx = 1.0f / cw;
    d.inv_cy = 1.0f / ch;
    T->set = true;
    return LIAR_OK;
}

extern "C" int liar_gpu_recovery_locate_device(liar_gpu_ctx* ctx, const float* d_xyz, size_t n, int32_t* d_idx,
                                               float* d_weights, void* stream) {
    if (!ctx) return LIAR_ERR_INVALID;
    if (n > 0 && (!d_xyz || !d_idx || !d_weights)) return ctx_fail(ctx, LIAR_ERR_INVALID, "null arrays");
    int rc = ctx_activate(ctx);
    if (rc) return rc;
    return recovery_locate_device(ctx, d_xyz, n, d_idx, d_weights, stream ? (cudaStream_t)stream : ctx->stream);
}
