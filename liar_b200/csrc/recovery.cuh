// recovery.cuh -- spectra of tristimulus values on the device: the reference's standard
// RecoveryMengSimon (src/liar/spectra/recovery_meng_simon.cpp:151-310) in Single mode.
//
// The table (set per context by liar_gpu_set_recovery): spectra sampled at chromaticities xy and
// a triangulation of those points plus the four corners of the box [-0.3, 1.0] x [-0.3, 1.2],
// whose corners carry the zero spectrum. A uniform grid over the box lists the triangles whose
// bounding box meets each cell, so that locating a chromaticity tests a few triangles.
#pragma once
#include <math.h>
#include <stdint.h>

namespace liar_gpu {

struct DRecovery {
    const float* wavelengths;  // n_w, metres, increasing
    const float* spectra;      // n_s x n_w
    const float* maxima;       // n_s
    const float* points;       // (n_s + 4) x 2: the samples, then the box corners
    const int32_t* tris;       // n_t x 3 point indices
    const int32_t* cell_first; // gx * gy + 1: the cell's range in cell_tris
    const int32_t* cell_tris;
    int n_w, n_s, n_t, gx, gy;
    float lo_x, lo_y, inv_cx, inv_cy;
};

constexpr float kRecoveryBoxLoX = -0.3f, kRecoveryBoxLoY = -0.3f, kRecoveryBoxHiX = 1.0f, kRecoveryBoxHiY = 1.2f;

// one colour's blend: up to three table spectra (index -1: zero spectrum) with their weights
struct RecoveryBlend {
    int32_t idx[3];
    float w[3];
};

#ifdef __CUDACC__
#define LIAR_REC_HD __host__ __device__
#else
#define LIAR_REC_HD
#endif

// RecoveryMengSimon::Impl::recover: false when the colour has no recovery (zero sum, chromaticity
// outside the box). The weights are barycentric in the containing triangle, zero at the box
// corners, then scaled to sum to X + Y + Z.
LIAR_REC_HD inline bool recovery_locate(const DRecovery& R, float X, float Y, float Z, RecoveryBlend& out) {
    const float s = X + Y + Z;
    if (s == 0.0f || R.n_t == 0) return false;
    const float x = X / s, y = Y / s;
    if (!(x >= kRecoveryBoxLoX && x <= kRecoveryBoxHiX && y >= kRecoveryBoxLoY && y <= kRecoveryBoxHiY)) return false;
    int cx = (int)((x - R.lo_x) * R.inv_cx), cy = (int)((y - R.lo_y) * R.inv_cy);
    cx = cx < 0 ? 0 : (cx >= R.gx ? R.gx - 1 : cx);
    cy = cy < 0 ? 0 : (cy >= R.gy ? R.gy - 1 : cy);
    const int cell = cy * R.gx + cx;
    int best = -1;
    float bw[3] = {0.0f, 0.0f, 0.0f}, best_min = -INFINITY;
    for (int k = R.cell_first[cell]; k < R.cell_first[cell + 1]; ++k) {
        const int t = R.cell_tris[k];
        const int i0 = R.tris[3 * t], i1 = R.tris[3 * t + 1], i2 = R.tris[3 * t + 2];
        const float ax = R.points[2 * i0], ay = R.points[2 * i0 + 1];
        const float bx = R.points[2 * i1], by = R.points[2 * i1 + 1];
        const float qx = R.points[2 * i2], qy = R.points[2 * i2 + 1];
        const float det = (bx - ax) * (qy - ay) - (qx - ax) * (by - ay);
        if (det == 0.0f) continue;
        const float w1 = ((x - ax) * (qy - ay) - (qx - ax) * (y - ay)) / det;
        const float w2 = ((bx - ax) * (y - ay) - (x - ax) * (by - ay)) / det;
        const float w0 = 1.0f - w1 - w2;
        const float mn = fminf(w0, fminf(w1, w2));
        // the containing triangle; on an edge either neighbour gives the same blend, and round-off
        // outside every triangle takes the least violated one
        if (mn > best_min) {
            best_min = mn;
            best = t;
            bw[0] = w0;
            bw[1] = w1;
            bw[2] = w2;
        }
        if (mn >= 0.0f) break;
    }
    if (best < 0) return false;
    float wtot = 0.0f;
    for (int j = 0; j < 3; ++j) {
        const int i = R.tris[3 * best + j];
        out.idx[j] = i < R.n_s ? i : -1;
        if (out.idx[j] < 0) bw[j] = 0.0f;
        wtot += bw[j];
    }
    if (wtot == 0.0f) return false;
    for (int j = 0; j < 3; ++j) out.w[j] = bw[j] * (s / wtot);
    return true;
}

// RecoveryMengSimon::doRecover (Single mode) at wavelength w: the blend interpolated linearly
// between the table's wavelengths, zero outside them; reflectant: divided by the blend of the
// maxima when that exceeds 1
LIAR_REC_HD inline float recovery_eval(const DRecovery& R, const RecoveryBlend& b, float w, bool reflectant) {
    const float* ws = R.wavelengths;
    int lo = 0, hi = R.n_w;  // first index with ws[k] > w
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (ws[mid] > w) hi = mid;
        else lo = mid + 1;
    }
    const int k = lo;
    if (k == 0 || k == R.n_w) return 0.0f;
    const float t = (w - ws[k - 1]) / (ws[k] - ws[k - 1]);
    float v0 = 0.0f, v1 = 0.0f, mx = 0.0f;
    for (int j = 0; j < 3; ++j) {
        if (b.idx[j] < 0) continue;
        const float* sp = R.spectra + (size_t)b.idx[j] * R.n_w;
        v0 += b.w[j] * sp[k - 1];
        v1 += b.w[j] * sp[k];
        mx += b.w[j] * R.maxima[b.idx[j]];
    }
    const float v = v0 + t * (v1 - v0);
    if (reflectant && mx > 1.0f) return v / mx;
    return v;
}

#undef LIAR_REC_HD

}  // namespace liar_gpu
