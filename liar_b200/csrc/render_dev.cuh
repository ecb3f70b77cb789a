// render_dev.cuh -- device-side shading of the spectral path tracer: spectra at one wavelength,
// the observer, the per-pixel stratified sampler, BSDFs, lights. Used by render.cu.
//
// Everything here restates the reference's per-sample arithmetic in single precision:
//   spectra    src/liar/kernel/spectral.cpp:178-220, spectra/sampled.cpp:128,
//              spectra/black_body.cpp:44-118, spectra/cauchy.cpp:72-76
//   observer   src/liar/kernel/observer.cpp:57-171, 283-317
//   BSDFs      src/liar/kernel/bsdf.cpp:52-98 (caps filtering), shaders/lambert.cpp:105-124,
//              conductor.cpp:179-196, cook_torrance.cpp:234-295, dielectric.cpp:148-245,
//              walter.cpp:215-415, mirror.cpp:142-160, kernel/microfacet.cpp:56-122,
//              shaders/microfacet_trowbridge_reitz.cpp:47-80, microfacet_beckmann.cpp:53-124
//   lights     src/liar/scenery/light_area.cpp:189-288, light_point.cpp:160-196,
//              light_sky.cpp:140-363, scenery/parallelogram.cpp, triangle_mesh.cpp:414-443,
//              kernel/scene_object.cpp (area to solid-angle pdf, angularPdf),
//              kernel/light_context.cpp:272-333 (power CDF)
// Lass routines the reference calls (cosineHemisphere, uniformSphere, uniformDisk) are restated
// from published methods: Malley's method on the Shirley-Chiu concentric disk mapping, the
// Archimedes cylinder map for the sphere.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/liar_gpu.h"
#include "recovery.cuh"
#include "qbvh.h"
#include "tri_exact.h"

namespace liar_gpu {
namespace rt {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kTol = 1e-6f;  // liar::tolerance (src/liar/kernel/kernel_common.cpp:32)
constexpr float kEps = 1.19209290e-07f;  // numeric_limits<float>::epsilon

enum : uint32_t { CAP_EMISSION = 0x1, CAP_REFL = 0x2, CAP_TRANS = 0x4, CAP_DIFF = 0x10, CAP_SPEC = 0x20,
                  CAP_GLOSSY = 0x40, CAP_ALL = 0xff };

__host__ __device__ __forceinline__ bool has_caps(uint32_t caps, uint32_t wanted) { return (caps & wanted) == wanted; }
__host__ __device__ __forceinline__ bool compatible_caps(uint32_t caps, uint32_t allowed) {
    const uint32_t o = caps & allowed;
    return (o & 0xf) > 0 && (o & 0xf0) > 0;
}

// ---- small vector helpers
__device__ __forceinline__ float3 mk(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return mk(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return mk(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float norm(float3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ float3 normal(float3 a) { return (1.0f / norm(a)) * a; }
__device__ __forceinline__ float sqr(float x) { return x * x; }
__device__ __forceinline__ float lerpf(float a, float b, float t) { return a + t * (b - a); }
// Lass Vector3D::reflect: mirror `v` about this (unit) normal h
__device__ __forceinline__ float3 reflect_about(float3 h, float3 v) { return (2.0f * dot(h, v)) * h - v; }

// ---- scene as the kernels see it
struct DScene {
    const QNode* nodes;
    const QTri* qtris;
    const float* verts;          // n x 3
    const uint32_t* tri_idx;     // n x 3
    const int32_t* tri_obj;
    const float* normals;        // optional
    const int32_t* tri_nrm;      // optional, n x 3
    const int32_t* obj_mat;
    const int32_t* obj_light;
    const liar_material* mats;
    const liar_spectrum* specs;
    const float* pool;
    const float* spec_max;       // per spectrum: max of a sampled spectrum's values (reflectant rescale)
    const liar_light* lights;
    const float* light_cdf;      // n_lights, normalised cumulative power
    const float* light_area;     // n_lights
    const float* tri_cdf;        // per triangle: cumulative area within its mesh light (normalised)
    int n_lights;
    const float* obs_w;          // n_obs
    const float* obs_xyz;        // n_obs x 3, normalised so that Y of the unit spectrum is 1
    const float* obs_dxyz;       // n_obs x 3, slope to the next sample
    const float* obs_cdf;        // n_obs
    int n_obs;
    float sky_distance;
    int sky_light;
    uint32_t stack_needed;
    const liar_texture* texs;    // optional texture nodes
    int n_tex;
    const float* tri_uv;         // optional, per triangle 3 x (u, v)
    const float4* tex_pixels;    // image textures' XYZ pixels
    const uint8_t* noise_tables; // noise textures' permutation tables
    DRecovery rec;               // the recovery of image pixels (set when the scene has images)
    const DScene* self;          // this description in device memory (for out-of-line lookups)
    const float4* spheres;       // analytic spheres: centre, radius; primitive n_tris + k
    const int32_t* sphere_obj;
    uint32_t n_tris;
};

// the object of a hit primitive (a triangle, or an analytic sphere past the triangles)
__device__ __forceinline__ int prim_object(const DScene& S, uint32_t prim) {
    return prim < S.n_tris ? S.tri_obj[prim] : S.sphere_obj[prim - S.n_tris];
}

// ---- spectra
__device__ __forceinline__ float planck(float w, float T) {
    const float h = 6.626070040e-34f, c = 299792458.0f, kb = 1.3806488e-23f;
    const float c1 = 2 * h * c * c, c2 = h * c / kb;
    const float w5 = sqr(sqr(w)) * w;
    return c1 / (w5 * expm1f(c2 / (w * T)));
}

__device__ __forceinline__ int upper_bound_f(const float* a, int n, float x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] > x) hi = mid; else lo = mid + 1;
    }
    return lo;
}
__device__ __forceinline__ int lower_bound_f(const float* a, int n, float x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// value of spectrum idx at wavelength w (m); reflectant spectra are clamped / rescaled to <= 1
// like Spectral(..., SpectralType::Reflectant) (src/liar/kernel/spectral.cpp:47-70, 185-210)
__device__ inline float spec_eval(const DScene& S, int idx, float w, bool reflectant) {
    if (idx < 0) return 0.0f;
    const liar_spectrum sp = S.specs[idx];
    float v;
    switch (sp.type) {
        case LIAR_SPEC_SAMPLED: {
            const float* ws = S.pool + sp.offset;
            const float* vs = ws + sp.count;
            const int i = upper_bound_f(ws, sp.count, w);
            if (i == 0 || i == sp.count) return 0.0f;
            const float t = (w - ws[i - 1]) / (ws[i] - ws[i - 1]);
            v = lerpf(vs[i - 1], vs[i], t);
            if (reflectant) {
                const float mx = S.spec_max[idx];
                if (mx > 1.0f) return v / mx;
            }
            return v;
        }
        case LIAR_SPEC_BLACKBODY: {
            const float T = sp.p[0];
            const float inv_norm = 1.0f / planck(2.897771955e-3f / T, T);
            v = sp.p[1] * inv_norm * planck(w, T);
            break;
        }
        case LIAR_SPEC_CAUCHY: {
            const float wu = w * 1e6f;
            v = sp.p[0] + sp.p[1] / sqr(wu);
            break;
        }
        default:
            v = sp.p[0];
    }
    return reflectant ? fminf(v, 1.0f) : v;
}

// ---- observer
__device__ inline float observer_sample(const DScene& S, float u, float& pdf) {
    const int n = S.n_obs;
    const int i = upper_bound_f(S.obs_cdf, n, u);
    if (i == 0 || i == n) {
        pdf = 0.0f;
        return i == 0 ? S.obs_w[0] : S.obs_w[n - 1];
    }
    const float c1 = S.obs_cdf[i - 1], c2 = S.obs_cdf[i];
    const float dc = c2 - c1;
    const float x = (u - c1) / dc;
    const float w1 = S.obs_w[i - 1], w2 = S.obs_w[i];
    pdf = dc / (w2 - w1);
    return lerpf(w1, w2, x);
}

__device__ inline float3 observer_sensitivity(const DScene& S, float w) {
    const int i = upper_bound_f(S.obs_w, S.n_obs, w);
    if (i == 0 || i == S.n_obs) return mk(0, 0, 0);
    const int k = i - 1;
    const float dw = w - S.obs_w[k];
    return mk(S.obs_xyz[3 * k] + S.obs_dxyz[3 * k] * dw, S.obs_xyz[3 * k + 1] + S.obs_dxyz[3 * k + 1] * dw,
              S.obs_xyz[3 * k + 2] + S.obs_dxyz[3 * k + 2] * dw);
}

// ---- sampler: per-pixel stratified dimensions (see sampler.h for the definition)
}  // namespace rt
}  // namespace liar_gpu

#include "sampler.h"

namespace liar_gpu {
namespace rt {

// Malley's method on the concentric disk (Shirley & Chiu 1997): cosine-weighted hemisphere
__device__ __forceinline__ float2 concentric_disk(float u1, float u2) {
    const float a = 2.0f * u1 - 1.0f, b = 2.0f * u2 - 1.0f;
    if (a == 0.0f && b == 0.0f) return make_float2(0.0f, 0.0f);
    float r, phi;
    if (fabsf(a) > fabsf(b)) {
        r = a;
        phi = (kPi / 4) * (b / a);
    } else {
        r = b;
        phi = (kPi / 2) - (kPi / 4) * (a / b);
    }
    return make_float2(r * cosf(phi), r * sinf(phi));
}
__device__ __forceinline__ float3 cosine_hemisphere(float u1, float u2, float& pdf) {
    const float2 d = concentric_disk(u1, u2);
    const float z = sqrtf(fmaxf(0.0f, 1.0f - d.x * d.x - d.y * d.y));
    pdf = z / kPi;
    return mk(d.x, d.y, z);
}
// Archimedes: z uniform in [-1, 1], phi uniform
__device__ __forceinline__ float3 uniform_sphere(float u1, float u2, float& pdf) {
    const float z = 1.0f - 2.0f * u2;
    const float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
    const float phi = 2.0f * kPi * u1;
    pdf = 1.0f / (4.0f * kPi);
    return mk(r * cosf(phi), r * sinf(phi), z);
}

// ---- BSDFs in the shading frame (z = shading normal)
struct Bsdf {
    uint32_t type;
    uint32_t caps;
    int mdf;
    float3 ng;          // geometric normal in the BSDF frame
    float r;            // diffuse / reflectance at the wavelength
    float t;            // transmittance (dielectrics)
    float eta, kappa;   // conductors
    float ior;          // dielectric: ratio used by DielectricBsdf
    float eta_i, eta_t; // Walter
    float au, av;       // microfacet alphas (roughness squared)
};

struct BsdfOut {
    float value, pdf;
};
struct BsdfSample {
    float3 wo;
    float value, pdf;
    __device__ bool ok() const { return pdf > 0.0f && value != 0.0f; }
};

__device__ __forceinline__ float power_heuristic(float a, float b) { return sqr(a) / (sqr(a) + sqr(b)); }

// microfacet distributions
__device__ inline float mdf_sample_phi(float s, float au, float av) {
    if (au == av) return 2 * kPi * s;
    const float phi = atanf(av / au * tanf(2 * kPi * s));
    if (s <= 0.25f) return phi;
    if (s < 0.75f) return phi + kPi;
    return phi + 2 * kPi;
}
__device__ inline float mdf_D(int mdf, float3 h, float au, float av, float& pdfH) {
    if (mdf == LIAR_MDF_GGX) {
        const float d = 1.0f / (kPi * au * av * sqr(sqr(h.x / au) + sqr(h.y / av) + sqr(h.z)));
        pdfH = d * h.z;
        return d;
    }
    const float c2 = sqr(h.z);
    if (c2 == 0.0f) {
        pdfH = 0.0f;  // the reference leaves pdfH untouched here; zero keeps the sample invalid
        return 0.0f;
    }
    const float d = expf(-(sqr(h.x / au) + sqr(h.y / av)) / c2) / (kPi * au * av * sqr(c2));
    pdfH = d * h.z;
    return d;
}
__device__ inline float3 mdf_sample_h(int mdf, float sx, float sy, float au, float av) {
    if (mdf == LIAR_MDF_GGX) {
        const float phi = mdf_sample_phi(sx, au, av);
        const float s = sqrtf(sy / (1.0f - sy));
        return normal(mk(s * au * cosf(phi), s * av * sinf(phi), 1.0f));
    }
    const float s = logf(1.0f - sx);
    float cp, sp, tan2;
    if (au == av) {
        const float phi = 2 * kPi * sy;
        cp = cosf(phi);
        sp = sinf(phi);
        tan2 = -s * sqr(au);
    } else {
        const float phi = mdf_sample_phi(sx, au, av);  // the reference reuses sample.x here
        cp = cosf(phi);
        sp = sinf(phi);
        tan2 = -s / (sqr(cp / au) + sqr(sp / av));
    }
    const float c2 = 1.0f / (1.0f + tan2);
    const float ct = sqrtf(c2);
    const float st = sqrtf(fmaxf(1.0f - c2, 0.0f));
    return mk(cp * st, sp * st, ct);
}
__device__ inline float mdf_lambda(int mdf, float3 w, float au, float av) {
    if (mdf == LIAR_MDF_GGX) {
        const float inv_a2 = (sqr(w.x * au) + sqr(w.y * av)) / sqr(w.z);
        return (sqrtf(1.0f + inv_a2) - 1.0f) / 2.0f;
    }
    // the reference's Beckmann Lambda returns this rational fit (microfacet_beckmann.cpp:110-124)
    const float a2 = sqr(w.z) / (sqr(w.x * au) + sqr(w.y * av));
    const float a = sqrtf(a2);
    return a < 1.6f ? (3.535f * a + 2.181f * a2) / (1.0f + 2.276f * a + 2.577f * a2) : 1.0f;
}
__device__ inline float mdf_G1(int mdf, float3 w, float3 h, float au, float av) {
    if (dot(w, h) * w.z <= 0.0f) return 0.0f;
    return 1.0f / (1.0f + mdf_lambda(mdf, w, au, av));
}

__device__ inline float fresnel_conductor(float eta, float kappa, float cosI) {
    const float c2 = sqr(cosI);
    const float a = sqr(eta) + sqr(kappa);
    const float b = (2 * cosI) * eta;
    const float aO = a + c2, aP = a * c2 + 1;
    return ((aO - b) / (aO + b) + (aP - b) / (aP + b)) / 2;
}
__device__ inline float fresnel_dielectric_walter(float ior, float3 wi, float3 h) {
    const float cosI = fabsf(dot(wi, h));
    const float sinT2 = sqr(ior) * (1 - sqr(cosI));
    const float cosT = sqrtf(fmaxf(1 - sinT2, 0.0f));
    const float rO = (ior * cosI - cosT) / (ior * cosI + cosT);
    const float rP = (cosI - ior * cosT) / (cosI + ior * cosT);
    return fminf((sqr(rO) + sqr(rP)) / 2, 1.0f);
}
__device__ inline float walter_pdf_reflection(const Bsdf& b, float rF, uint32_t allowed) {
    const float pr = has_caps(allowed, CAP_REFL | CAP_GLOSSY) ? fabsf(b.r) * rF : 0.0f;
    const float pt = has_caps(allowed, CAP_TRANS | CAP_GLOSSY) ? fabsf(b.t) * (1 - rF) : 0.0f;
    const float tot = pr + pt;
    if (tot == 0.0f) return -1.0f;
    return pr / tot;
}

__device__ inline BsdfOut bsdf_do_evaluate(const Bsdf& b, float3 wi, float3 wo, uint32_t allowed) {
    BsdfOut out{0.0f, 0.0f};
    switch (b.type) {
        case LIAR_MAT_LAMBERT: {
            const float c = fabsf(wo.z);
            if (c <= 0.0f) return out;
            return BsdfOut{b.r / kPi, c / kPi};
        }
        case LIAR_MAT_COOK_TORRANCE: {
            if (wo.z <= 0.0f) return out;
            const float3 h = normal(wi + wo);
            float pdfH;
            const float d = mdf_D(b.mdf, h, b.au, b.av, pdfH);
            const float dh = fabsf(dot(wi, h));
            const float g = fminf(1.0f, fminf(2 * h.z * wi.z / dh, 2 * h.z * wo.z / dh));
            const float pdf = pdfH / (4 * dot(wi, h));
            float v = b.r * (d * g / (4 * wi.z * wo.z));
            v *= fresnel_conductor(b.eta, b.kappa, fabsf(dot(wi, h)));
            return BsdfOut{v, pdf};
        }
        case LIAR_MAT_WALTER: {
            if (wo.z > 0.0f) {
                const float3 h = normal(wi + wo);
                const float rF = fresnel_dielectric_walter(b.eta_i / b.eta_t, wi, h);
                const float pR = walter_pdf_reflection(b, rF, allowed);
                if (pR < 0.0f) return out;
                float pdfH;
                const float d = mdf_D(b.mdf, h, b.au, b.av, pdfH);
                const float g = mdf_G1(b.mdf, wi, h, b.au, b.av) * mdf_G1(b.mdf, wo, h, b.au, b.av);
                const float dh = 1.0f / (4 * dot(wi, h));
                return BsdfOut{b.r * (rF * d * g / (4 * wi.z * wo.z)), pR * pdfH * dh};
            } else if (wo.z < 0.0f) {
                const float3 h = normal(-(b.eta_i * wi) - b.eta_t * wo);
                if (h.z <= 0.0f) return out;
                const float cI = fabsf(dot(wi, h)), cT = fabsf(dot(wo, h));
                const float rF = fresnel_dielectric_walter(b.eta_i / b.eta_t, wi, h);
                const float pR = walter_pdf_reflection(b, rF, allowed);
                if (pR < 0.0f) return out;
                float pdfH;
                const float d = mdf_D(b.mdf, h, b.au, b.av, pdfH);
                const float g = mdf_G1(b.mdf, wi, h, b.au, b.av) * mdf_G1(b.mdf, wo, h, b.au, b.av);
                const float dh = sqr(b.eta_t) * cT / sqr(b.eta_i * cI + b.eta_t * cT);
                return BsdfOut{b.t * (((1 - rF) * d * g * (cI * dh)) / fabsf(wi.z * wo.z)), (1 - pR) * pdfH * dh};
            }
            return out;
        }
        default:  // specular BSDFs have no finite density
            return out;
    }
}

// Bsdf::evaluate: reject wo in the plane, drop the caps that the geometric normal rules out
__device__ inline BsdfOut bsdf_evaluate(const Bsdf& b, float3 wi, float3 wo, uint32_t allowed) {
    if (wo.z == 0.0f) return BsdfOut{0.0f, 0.0f};
    const bool reflective = (dot(wi, b.ng) > 0.0f) == (dot(wo, b.ng) > 0.0f);
    allowed &= ~(reflective ? CAP_TRANS : CAP_REFL);
    if (!compatible_caps(b.caps, allowed)) return BsdfOut{0.0f, 0.0f};
    return bsdf_do_evaluate(b, wi, wo, allowed);
}

__device__ inline BsdfSample bsdf_sample(const Bsdf& b, float3 wi, float sx, float sy, float comp, uint32_t allowed) {
    BsdfSample out{mk(0, 0, 0), 0.0f, 0.0f};
    if (!compatible_caps(b.caps, allowed)) return out;
    switch (b.type) {
        case LIAR_MAT_LAMBERT: {
            float pdf;
            out.wo = cosine_hemisphere(sx, sy, pdf);
            out.pdf = pdf;
            out.value = b.r / kPi;
            return out;
        }
        case LIAR_MAT_CONDUCTOR: {
            const float cosI = wi.z;
            out.wo = mk(-wi.x, -wi.y, wi.z);
            out.value = b.r * fresnel_conductor(b.eta, b.kappa, cosI) / cosI;
            out.pdf = 1.0f;
            return out;
        }
        case LIAR_MAT_MIRROR: {
            out.wo = mk(-wi.x, -wi.y, wi.z);
            out.value = b.r;
            out.pdf = out.wo.z;
            return out;
        }
        case LIAR_MAT_COOK_TORRANCE: {
            const float3 h = mdf_sample_h(b.mdf, sx, sy, b.au, b.av);
            const float3 wo = reflect_about(h, wi);
            if (wo.z <= 0.0f) return out;
            const BsdfOut e = bsdf_do_evaluate(b, wi, wo, allowed);
            out.wo = wo;
            out.value = e.value;
            out.pdf = e.pdf;
            return out;
        }
        case LIAR_MAT_DIELECTRIC: {
            const float cosI = wi.z;
            if (cosI <= 0.0f) return out;
            const float ior = b.ior;
            const float sinT2 = sqr(ior) * (1 - sqr(cosI));
            const float cosT = sqrtf(fmaxf(1 - sinT2, 0.0f));
            const float rO = (ior * cosI - cosT) / (ior * cosI + cosT);
            const float rP = (cosI - ior * cosT) / (cosI + ior * cosT);
            const float rF = (sqr(rO) + sqr(rP)) / 2;
            const float pr = has_caps(allowed, CAP_REFL | CAP_SPEC) ? fabsf(b.r) * rF : 0.0f;
            const float pt = has_caps(allowed, CAP_TRANS | CAP_SPEC) ? fabsf(b.t) * (1 - rF) : 0.0f;
            if (pr + pt == 0.0f) return out;
            const float probR = pr / (pr + pt);
            if (comp < probR) {
                out.wo = mk(-wi.x, -wi.y, wi.z);
                out.value = b.r * rF / cosI;
                out.pdf = probR;
            } else {
                out.wo = mk(-ior * wi.x, -ior * wi.y, -cosT);
                out.value = b.t * (1 - rF) / cosT;
                out.pdf = 1 - probR;
            }
            return out;
        }
        case LIAR_MAT_WALTER: {
            const float3 h = mdf_sample_h(b.mdf, sx, sy, b.au, b.av);
            float pdfH;
            const float d = mdf_D(b.mdf, h, b.au, b.av, pdfH);
            const float rF = fresnel_dielectric_walter(b.eta_i / b.eta_t, wi, h);
            const float pR = walter_pdf_reflection(b, rF, allowed);
            if (pR < 0.0f) return out;
            if (comp < pR) {
                const float3 wo = reflect_about(h, wi);
                if (wo.z <= 0.0f) return out;
                const float g = mdf_G1(b.mdf, wi, h, b.au, b.av) * mdf_G1(b.mdf, wo, h, b.au, b.av);
                const float dh = 1.0f / (4 * dot(wo, h));
                out.wo = wo;
                out.pdf = pR * pdfH * dh;
                out.value = b.r * (rF * d * g / (4 * wi.z * wo.z));
            } else {
                const float eta = b.eta_i / b.eta_t;
                const float cI = fabsf(dot(wi, h));
                const float s2 = sqr(eta) * (1 - sqr(cI));
                const float cT = sqrtf(fmaxf(1 - s2, 0.0f));
                const float3 wo = normal((-eta) * wi + (eta * cI - cT) * h);
                if (wo.z >= 0.0f) return out;
                const float g = mdf_G1(b.mdf, wi, h, b.au, b.av) * mdf_G1(b.mdf, wo, h, b.au, b.av);
                const float dh = sqr(b.eta_t) * cT / sqr(b.eta_i * cI + b.eta_t * cT);
                out.wo = wo;
                out.pdf = (1 - pR) * pdfH * dh;
                out.value = b.t * (((1 - rF) * d * g * (cI * dh)) / fabsf(wi.z * wo.z));
            }
            return out;
        }
        default:
            return out;
    }
}

// ---- lights
struct LightEmission {
    float value;   // radiance (unused by the light-sampling pdf sums)
    float pdf;     // solid-angle pdf of sampling this direction on this light
    float t;       // distance along the ray
};

// Parallelogram ray test (two-sided) for the light's surface; t in units of |d|, t > tmin
__device__ inline bool parallelogram_hit(const liar_light& L, float3 o, float3 d, float tmin, float& t) {
    const float3 p = mk(L.pos[0], L.pos[1], L.pos[2]), u = mk(L.u[0], L.u[1], L.u[2]), v = mk(L.v[0], L.v[1], L.v[2]);
    const float3 n = cross(u, v);
    const float den = dot(n, d);
    if (den == 0.0f) return false;
    const float th = dot(n, p - o) / den;
    if (!(th > tmin)) return false;
    const float3 x = o + th * d - p;
    // coordinates in the (u, v) basis
    const float uu = dot(u, u), uv = dot(u, v), vv = dot(v, v);
    const float xu = dot(x, u), xv = dot(x, v);
    const float det = uu * vv - uv * uv;
    const float a = (xu * vv - xv * uv) / det, b = (xv * uu - xu * uv) / det;
    if (a < 0.0f || a > 1.0f || b < 0.0f || b > 1.0f) return false;
    t = th;
    return true;
}

// SceneLight::emission for a ray leaving `o` along unit `d` (LightArea::doEmission ->
// SceneObject::doAngularPdf: t^2 / |A cos|; the single-sided test sees a normal already flipped
// toward the ray's origin, so hits are accepted from both sides)
__device__ inline LightEmission light_emission(const DScene& S, int li, float3 o, float3 d, float lambda) {
    LightEmission e{0.0f, 0.0f, INFINITY};
    const liar_light L = S.lights[li];
    if (L.type == LIAR_LIGHT_AREA_PARALLELOGRAM) {
        float t;
        if (!parallelogram_hit(L, o, d, kTol, t)) return e;
        const float3 n = normal(cross(mk(L.u[0], L.u[1], L.u[2]), mk(L.v[0], L.v[1], L.v[2])));
        e.pdf = sqr(t) / fabsf(S.light_area[li] * dot(d, n));
        e.t = t;
        e.value = spec_eval(S, L.spectrum, lambda, false);
        return e;
    }
    if (L.type == LIAR_LIGHT_AREA_MESH) {
        float tbest = INFINITY;
        int best = -1;
        for (int k = 0; k < L.n_tris; ++k) {
            const int ti = L.first_tri + k;
            const float* a = S.verts + 3 * S.tri_idx[3 * ti];
            const float* b = S.verts + 3 * S.tri_idx[3 * ti + 1];
            const float* c = S.verts + 3 * S.tri_idx[3 * ti + 2];
            float t, uu, vv;
            if (tri_intersect_exact(o.x, o.y, o.z, d.x, d.y, d.z, a[0], a[1], a[2], b[0] - a[0], b[1] - a[1],
                                    b[2] - a[2], c[0] - a[0], c[1] - a[1], c[2] - a[2], t, uu, vv) &&
                t > kTol && t < tbest) {
                tbest = t;
                best = ti;
            }
        }
        if (best < 0) return e;
        const float* a = S.verts + 3 * S.tri_idx[3 * best];
        const float* b = S.verts + 3 * S.tri_idx[3 * best + 1];
        const float* c = S.verts + 3 * S.tri_idx[3 * best + 2];
        const float3 n = normal(cross(mk(b[0] - a[0], b[1] - a[1], b[2] - a[2]), mk(c[0] - a[0], c[1] - a[1], c[2] - a[2])));
        e.pdf = sqr(tbest) / fabsf(S.light_area[li] * dot(d, n));
        e.t = tbest;
        e.value = spec_eval(S, L.spectrum, lambda, false);
        return e;
    }
    if (L.type == LIAR_LIGHT_SKY) {
        e.pdf = 1.0f / (4.0f * kPi);
        e.t = S.sky_distance;
        e.value = spec_eval(S, L.spectrum, lambda, false);
        return e;
    }
    return e;  // point lights are never hit
}

struct LightSample {
    float3 dir;
    float dist;
    float pdf;
    float value;
};

// SceneLight::sampleEmission(sample, lightSample, target, shadowRay, pdf)
__device__ inline LightSample light_sample(const DScene& S, int li, float3 target, float sx, float sy, float lambda) {
    LightSample out{mk(0, 0, 1), 0.0f, 0.0f, 0.0f};
    const liar_light L = S.lights[li];
    if (L.type == LIAR_LIGHT_AREA_PARALLELOGRAM || L.type == LIAR_LIGHT_AREA_MESH) {
        float3 p, n;
        float pdf;
        if (L.type == LIAR_LIGHT_AREA_PARALLELOGRAM) {
            const float3 u = mk(L.u[0], L.u[1], L.u[2]), v = mk(L.v[0], L.v[1], L.v[2]);
            p = mk(L.pos[0], L.pos[1], L.pos[2]) + sx * u + sy * v;
            n = normal(cross(u, v));
            pdf = 1.0f / S.light_area[li];
        } else {
            // TriangleMesh::doSampleSurface: pick a triangle by area, then a uniform point on it
            const float* cdf = S.tri_cdf + L.first_tri;
            int ii = lower_bound_f(cdf, L.n_tris, sx);
            if (ii > L.n_tris - 1) ii = L.n_tris - 1;
            const float i0 = ii > 0 ? cdf[ii - 1] : 0.0f;
            const float tpdf = cdf[ii] - i0;
            const float di = (sx - i0) / tpdf;
            const int ti = L.first_tri + ii;
            const float* a = S.verts + 3 * S.tri_idx[3 * ti];
            const float* b = S.verts + 3 * S.tri_idx[3 * ti + 1];
            const float* c = S.verts + 3 * S.tri_idx[3 * ti + 2];
            const float3 A = mk(a[0], a[1], a[2]);
            const float3 e1 = mk(b[0] - a[0], b[1] - a[1], b[2] - a[2]), e2 = mk(c[0] - a[0], c[1] - a[1], c[2] - a[2]);
            const float3 nn = cross(e1, e2);
            const float s = sqrtf(di);
            const float uu = 1.0f - s, vv = s * sy;
            const float nl = norm(nn);
            n = (1.0f / nl) * nn;
            pdf = tpdf / (nl / 2);
            p = A + uu * e1 + vv * e2;
        }
        // SceneObject::doSampleSurface(sample, target, ...): area pdf to solid angle
        float3 to = p - target;
        const float d2 = dot(to, to);
        to = (1.0f / sqrtf(d2)) * to;
        pdf *= d2 / fabsf(dot(n, to));
        // LightArea::doSampleEmission
        float3 tl = p - target;
        const float dist = norm(tl);
        tl = (1.0f / dist) * tl;
        out.dir = tl;
        out.dist = dist;
        if (!L.double_sided && dot(n, tl) > 0.0f) return out;  // target behind a single-sided light
        out.pdf = pdf;
        out.value = spec_eval(S, L.spectrum, lambda, false);
        return out;
    }
    if (L.type == LIAR_LIGHT_POINT) {
        float3 tl = mk(L.pos[0], L.pos[1], L.pos[2]) - target;
        const float d2 = dot(tl, tl);
        const float dist = sqrtf(d2);
        out.dir = (1.0f / dist) * tl;
        out.dist = dist;
        out.pdf = 1.0f;
        out.value = spec_eval(S, L.spectrum, lambda, false) / d2;  // default attenuation 1/d^2
        return out;
    }
    if (L.type == LIAR_LIGHT_SKY) {
        float pdf;
        out.dir = uniform_sphere(sx, sy, pdf);
        out.dist = S.sky_distance;
        out.pdf = pdf;
        out.value = spec_eval(S, L.spectrum, lambda, false);
        return out;
    }
    return out;
}

__device__ __forceinline__ float light_choice_pdf(const DScene& S, int k) {
    return k > 0 ? S.light_cdf[k] - S.light_cdf[k - 1] : S.light_cdf[0];
}

// ---- the local context of a hit (IntersectionContext, kernel/intersection_context.cpp:55-290)
struct HitContext {
    float3 target;  // hit point on the triangle
    float3 ng;      // geometric normal, flipped toward -d
    float3 N;       // shading normal, flipped toward -d
    float3 u, v;    // shading frame tangents
    bool leaving;   // solid event from the unflipped geometric normal
    int obj, light, mat;
    float uv_u, uv_v;  // surface coordinates: the triangle corners' (u, v) at the barycentrics, or those
    // screen-space footprint (IntersectionContext::dUv_dI / dUv_dJ and the larger squared norm of
    // dPoint_dI, dPoint_dJ): zero unless the hit carries ray differentials (hit_footprint)
    float du_i = 0.0f, dv_i = 0.0f, du_j = 0.0f, dv_j = 0.0f, fp2 = 0.0f;
};

__device__ inline HitContext hit_context(const DScene& S, float3 o, float3 d, uint32_t prim, float t) {
    HitContext H;
    if (prim >= S.n_tris) {
        // Sphere::doLocalContext (sphere.cpp:130-175): the point reprojected onto the surface, the
        // outward normal, uv from its spherical angles, dPoint/du along (-n.y, n.x, 0)
        const float4 sp = S.spheres[prim - S.n_tris];
        H.obj = S.sphere_obj[prim - S.n_tris];
        H.light = S.obj_light[H.obj];
        H.mat = S.obj_mat[H.obj];
        const float3 c = mk(sp.x, sp.y, sp.z);
        const float3 n0 = normal(o + t * d - c);
        H.target = c + sp.w * n0;
        H.uv_u = atan2f(n0.y, n0.x) * (0.5f / 3.14159265358979323846f);
        H.uv_v = acosf(fminf(fmaxf(n0.z, -1.0f), 1.0f)) * (1.0f / 3.14159265358979323846f);
        H.leaving = dot(d, n0) > 0.0f;
        H.ng = dot(n0, -1.0f * d) < 0.0f ? -1.0f * n0 : n0;
        H.N = H.ng;
        float3 u = mk(-n0.y, n0.x, 0.0f);
        u = u - dot(u, H.N) * H.N;
        if (dot(u, u) < 1e-12f) {
            const float3 ax = fabsf(H.N.x) < 0.9f ? mk(1, 0, 0) : mk(0, 1, 0);
            u = cross(ax, H.N);
        }
        H.u = normal(u);
        H.v = cross(H.N, H.u);
        return H;
    }
    H.obj = S.tri_obj[prim];
    H.light = S.obj_light[H.obj];
    H.mat = S.obj_mat[H.obj];
    // re-intersect the hit triangle for the barycentrics (TriangleMesh::doLocalContext)
    const uint32_t i0 = S.tri_idx[3 * prim], i1 = S.tri_idx[3 * prim + 1], i2 = S.tri_idx[3 * prim + 2];
    const float3 a = mk(S.verts[3 * i0], S.verts[3 * i0 + 1], S.verts[3 * i0 + 2]);
    const float3 b = mk(S.verts[3 * i1], S.verts[3 * i1 + 1], S.verts[3 * i1 + 2]);
    const float3 c = mk(S.verts[3 * i2], S.verts[3 * i2 + 1], S.verts[3 * i2 + 2]);
    const float3 e1 = b - a, e2 = c - a;
    float tt, bu, bv;
    if (!tri_intersect_exact(o.x, o.y, o.z, d.x, d.y, d.z, a.x, a.y, a.z, e1.x, e1.y, e1.z, e2.x, e2.y, e2.z, tt, bu, bv))
        bu = bv = 0.0f;
    H.target = a + bu * e1 + bv * e2;
    if (S.tri_uv) {
        const float* t = S.tri_uv + 6 * (size_t)prim;
        const float w0 = 1.0f - bu - bv;
        H.uv_u = w0 * t[0] + bu * t[2] + bv * t[4];
        H.uv_v = w0 * t[1] + bu * t[3] + bv * t[5];
    } else {
        H.uv_u = bu;
        H.uv_v = bv;
    }
    const float3 ng0 = normal(cross(e1, e2));
    float3 ns = ng0;
    if (S.tri_nrm) {
        const int n0 = S.tri_nrm[3 * prim], n1 = S.tri_nrm[3 * prim + 1], n2 = S.tri_nrm[3 * prim + 2];
        if (n0 >= 0 && n1 >= 0 && n2 >= 0) {
            const float w0 = 1.0f - bu - bv;
            ns = normal(w0 * mk(S.normals[3 * n0], S.normals[3 * n0 + 1], S.normals[3 * n0 + 2]) +
                        bu * mk(S.normals[3 * n1], S.normals[3 * n1 + 1], S.normals[3 * n1 + 2]) +
                        bv * mk(S.normals[3 * n2], S.normals[3 * n2 + 1], S.normals[3 * n2 + 2]));
        }
    }
    H.leaving = dot(d, ng0) > 0.0f;  // triangle_mesh.cpp:303-308
    H.ng = dot(ng0, -d) < 0.0f ? -ng0 : ng0;  // flipTo(-direction)
    H.N = dot(ns, -d) < 0.0f ? -ns : ns;
    // shading frame (IntersectionContext::bsdfToLocal)
    float3 u = e1 - dot(e1, H.N) * H.N;
    float3 v = e2 - dot(e2, H.N) * H.N;
    const float su = dot(u, u), sv = dot(v, v);
    if (fmaxf(su, sv) < 1e-3f * fmaxf(dot(e1, e1), dot(e2, e2))) {
        const float3 ax = fabsf(H.N.x) < 0.9f ? mk(1, 0, 0) : mk(0, 1, 0);
        u = cross(ax, H.N);
        v = cross(H.N, u);
    }
    if (su >= sv) {
        u = normal(u);
        v = cross(H.N, u);
    } else {
        v = normal(v);
        u = cross(v, H.N);
    }
    H.u = u;
    H.v = v;
    return H;
}

// Image::lookUp at mip level 0 (textures/image.cpp:654-718, 598-609): (u, 1 - v) over the
// pixels with wrap-around, nearest or bilinear between pixel centres; the indices are clamped
// where float rounding puts a wrapped coordinate on the image's far edge
// Perlin::noise (perlin.cpp:60-90, 170-205): improved Perlin noise over a 256-periodic lattice,
// gradients picked by the xor of three permutation tables (257 entries each, the last repeating
// the first), quintic fade, trilinear blend
__device__ inline float perlin_gradient(const uint8_t* tab, int x, int y, int z, float dx, float dy, float dz) {
    switch ((tab[x] ^ tab[257 + y] ^ tab[514 + z]) & 15) {
        case 0: return dx + dy;
        case 1: return dy - dx;
        case 2: return dx - dy;
        case 3: return -dx - dy;
        case 4: return dx + dz;
        case 5: return dz - dx;
        case 6: return dx - dz;
        case 7: return -dx - dz;
        case 8: return dy + dz;
        case 9: return dz - dy;
        case 10: return dy - dz;
        case 11: return -dy - dz;
        case 12: return dx + dy;
        case 13: return dy - dx;
        case 14: return dz - dy;
        default: return -dy - dz;
    }
}

__device__ __forceinline__ float perlin_fade(float d) {
    const float d2 = d * d;
    return (6.0f * d2 * d - 15.0f * d2 + 10.0f * d) * d2;
}

__device__ inline float perlin_noise(const uint8_t* tab, float3 q) {
    float c[3] = {q.x, q.y, q.z}, d[3];
    int i[3];
    for (int k = 0; k < 3; ++k) {
        const float m = c[k] - floorf(c[k] * (1.0f / 256.0f)) * 256.0f;  // num::mod(x, 256)
        const float f = floorf(m);
        i[k] = (int)f;
        d[k] = m - f;
        if (i[k] >= 256) i[k] = 0;  // rounding onto the period: the same lattice point as 0
        if (i[k] < 0) i[k] = 0;
    }
    const float g0 = perlin_gradient(tab, i[0], i[1], i[2], d[0], d[1], d[2]);
    const float g1 = perlin_gradient(tab, i[0] + 1, i[1], i[2], d[0] - 1, d[1], d[2]);
    const float g2 = perlin_gradient(tab, i[0], i[1] + 1, i[2], d[0], d[1] - 1, d[2]);
    const float g3 = perlin_gradient(tab, i[0] + 1, i[1] + 1, i[2], d[0] - 1, d[1] - 1, d[2]);
    const float g4 = perlin_gradient(tab, i[0], i[1], i[2] + 1, d[0], d[1], d[2] - 1);
    const float g5 = perlin_gradient(tab, i[0] + 1, i[1], i[2] + 1, d[0] - 1, d[1], d[2] - 1);
    const float g6 = perlin_gradient(tab, i[0], i[1] + 1, i[2] + 1, d[0], d[1] - 1, d[2] - 1);
    const float g7 = perlin_gradient(tab, i[0] + 1, i[1] + 1, i[2] + 1, d[0] - 1, d[1] - 1, d[2] - 1);
    const float sx = perlin_fade(d[0]), sy = perlin_fade(d[1]), sz = perlin_fade(d[2]);
    auto lerp = [](float a, float b, float t) { return a + t * (b - a); };
    return lerp(lerp(lerp(g0, g1, sx), lerp(g2, g3, sx), sy), lerp(lerp(g4, g5, sx), lerp(g6, g7, sx), sy), sz);
}

// the point a texture is looked up at: (u, v) with its screen-space derivatives, the squared
// footprint on the surface (FBm's octave count) and the hit point (noise textures)
struct TexPoint {
    float u, v, du_i, dv_i, du_j, dv_j, fp2;
    float3 x;
};

// CheckerBoard::weightA (checker_board.cpp:149-181): 1 or 0 without anti-aliasing; with bilinear
// anti-aliasing the share of A over the footprint's (u, v) box, half a derivative to each side
// (CheckerBoard::integrate, checker_board.cpp:185-207), the point rule where the box is empty
__device__ inline float checker_weight(const liar_texture& T, const TexPoint& q) {
    const float sx = T.p[0], sy = T.p[1];
    const float fu = q.u - floorf(q.u), fv = q.v - floorf(q.v);
    const float point = (fu < sx) == (fv < sy) ? 1.0f : 0.0f;
    if (T.p[2] == 0.0f) return point;
    const float du = fmaxf(fabsf(q.du_i), fabsf(q.du_j)), dv = fmaxf(fabsf(q.dv_i), fabsf(q.dv_j));
    const float area = du * dv;
    if (!(area > 0.0f)) return point;
    const float mnu = fu - du / 2, mnv = fv - dv / 2, mxu = fu + du / 2, mxv = fv + dv / 2;
    const float mn0u = floorf(mnu), mn0v = floorf(mnv), mx0u = floorf(mxu), mx0v = floorf(mxv);
    const float d0u = mx0u - mn0u, d0v = mx0v - mn0v;
    const float dmnu = mnu - mn0u, dmnv = mnv - mn0v, dmxu = mxu - mx0u, dmxv = mxv - mx0v;
    // (min(d, split), max(d - split, 0)) per corner and axis
    const float mnU0 = fminf(dmnu, sx), mnU1 = fmaxf(dmnu - sx, 0.0f);
    const float mnV0 = fminf(dmnv, sy), mnV1 = fmaxf(dmnv - sy, 0.0f);
    const float mxU0 = fminf(dmxu, sx), mxU1 = fmaxf(dmxu - sx, 0.0f);
    const float mxV0 = fminf(dmxv, sy), mxV1 = fmaxf(dmxv - sy, 0.0f);
    const float oneU0 = sx, oneU1 = 1.0f - sx, oneV0 = sy, oneV1 = 1.0f - sy;
    float r = (sx * sy + (1.0f - sx) * (1.0f - sy)) * d0u * d0v;
    r += ((oneU0 * mxV0 + oneU1 * mxV1) - (oneU0 * mnV0 + oneU1 * mnV1)) * d0u;
    r += ((mxU0 * oneV0 + mxU1 * oneV1) - (mnU0 * oneV0 + mnU1 * oneV1)) * d0v;
    r += (mxU0 * mxV0 + mxU1 * mxV1) - (mxU0 * mnV0 + mxU1 * mnV1);
    r += (mnU0 * mnV0 + mnU1 * mnV1) - (mnU0 * mxV0 + mnU1 * mxV1);
    return fminf(fmaxf(r / area, 0.0f), 1.0f);
}

// Image::mipMapLevel (image.cpp:580-612): the level of a footprint `width` in (u or v) units is
// maxLevel + log2(width), its fraction from the significand (log2(m) ~ m - 1 for 1 <= m < 2)
__device__ inline void mip_level(float width, int n_levels, int& l0, int& l1, float& frac) {
    const int max_level = n_levels - 1;
    const float w = fmaxf(width, 1e-9f);
    const int i = __float_as_int(w);
    const int level = max_level + ((i >> 23) - 127);
    if (level < 0) {
        l0 = l1 = 0;
        frac = 0.0f;
    } else if (level >= max_level) {
        l0 = l1 = max_level;
        frac = 0.0f;
    } else {
        l0 = level;
        l1 = level + 1;
        frac = __int_as_float((127 << 23) | (i & 0x7fffff)) - 1.0f;
    }
}

// one level of an image's mip table (the header at `pixels`: level counts, then per level the
// offset of its pixels and its size; textures.Image lays it out)
struct MipLevel {
    const float4* px;
    int w, h;
};
__device__ __forceinline__ MipLevel mip_get(const DScene& S, const liar_texture& T, int n_u, int iu, int iv) {
    const float4* base = S.tex_pixels + T.pixels;
    const float4 e = base[1 + iv * n_u + iu];
    MipLevel m;
    m.px = base + ((int64_t)__float_as_int(e.y) << 31 | (int64_t)(uint32_t)__float_as_int(e.x));
    m.w = __float_as_int(e.z);
    m.h = __float_as_int(e.w);
    return m;
}

// Image::nearest (image.cpp:618-631): the pixel under (u, 1 - v), wrapped
__device__ inline float3 image_nearest(const MipLevel& m, float u, float v) {
    const float w = 1.0f - v;
    int x0 = (int)floorf((u - floorf(u)) * (float)m.w);
    int y0 = (int)floorf((w - floorf(w)) * (float)m.h);
    x0 = min(max(x0, 0), m.w - 1);
    y0 = min(max(y0, 0), m.h - 1);
    const float4 p = m.px[(size_t)y0 * m.w + x0];
    return mk(p.x, p.y, p.z);
}

// Image::bilinear (image.cpp:636-690, the vectorised build): the fractional (u, 1 - v) scaled to
// the level, half a pixel back, the four neighbours with wrap-around
__device__ inline float3 image_bilinear(const MipLevel& m, float u, float v) {
    const float w = 1.0f - v;
    const float x = (u - floorf(u)) * (float)m.w - 0.5f, y = (w - floorf(w)) * (float)m.h - 0.5f;
    const float x0 = floorf(x), y0 = floorf(y);
    const float dx = x - x0, dy = y - y0;
    int i0 = (int)x0, j0 = (int)y0;
    if (i0 < 0) i0 += m.w;
    if (j0 < 0) j0 += m.h;
    i0 = min(max(i0, 0), m.w - 1);
    j0 = min(max(j0, 0), m.h - 1);
    const int i1 = i0 + 1 < m.w ? i0 + 1 : 0, j1 = j0 + 1 < m.h ? j0 + 1 : 0;
    const float4 p00 = m.px[(size_t)j0 * m.w + i0], p10 = m.px[(size_t)j0 * m.w + i1];
    const float4 p01 = m.px[(size_t)j1 * m.w + i0], p11 = m.px[(size_t)j1 * m.w + i1];
    const float ex = 1.0f - dx, ey = 1.0f - dy;
    const float3 a = mk(ex * p00.x + dx * p10.x, ex * p00.y + dx * p10.y, ex * p00.z + dx * p10.z);
    const float3 b = mk(ex * p01.x + dx * p11.x, ex * p01.y + dx * p11.y, ex * p01.z + dx * p11.z);
    return mk(ey * a.x + dy * b.x, ey * a.y + dy * b.y, ey * a.z + dy * b.z);
}

// Image::lookUp (image.cpp:249-330): mip levels from the footprint (none: level 0; isotropic: the
// largest derivative over one chain of levels; anisotropic: u and v derivatives over a table of
// levels), then nearest, bilinear, or trilinear (bilinear lookups blended across the levels)
__device__ inline float3 image_lookup(const DScene& S, const liar_texture& T, const TexPoint& q) {
    const float4 hdr = S.tex_pixels[T.pixels];
    const int n_u = __float_as_int(hdr.x), n_v = __float_as_int(hdr.y), mip = __float_as_int(hdr.z);
    int u0 = 0, u1 = 0, v0 = 0, v1 = 0;
    float fu = 0.0f, fv = 0.0f;
    const float wu = fmaxf(fabsf(q.du_i), fabsf(q.du_j)), wv = fmaxf(fabsf(q.dv_i), fabsf(q.dv_j));
    if (mip == 1) {
        mip_level(fmaxf(wu, wv), n_u, u0, u1, fu);
    } else if (mip == 2) {
        mip_level(wu, n_u, u0, u1, fu);
        mip_level(wv, n_v, v0, v1, fv);
    }
    const int aa = (int)T.p[0];
    if (aa == 0) return image_nearest(mip_get(S, T, n_u, u0, v0), q.u, q.v);
    if (aa == 1) return image_bilinear(mip_get(S, T, n_u, u0, v0), q.u, q.v);
    const float3 p00 = image_bilinear(mip_get(S, T, n_u, u0, v0), q.u, q.v);
    const float3 p10 = image_bilinear(mip_get(S, T, n_u, u1, v0), q.u, q.v);
    const float eu = 1.0f - fu;
    float3 r = mk(eu * p00.x + fu * p10.x, eu * p00.y + fu * p10.y, eu * p00.z + fu * p10.z);
    if (v0 != v1) {
        const float3 p01 = image_bilinear(mip_get(S, T, n_u, u0, v1), q.u, q.v);
        const float3 p11 = image_bilinear(mip_get(S, T, n_u, u1, v1), q.u, q.v);
        const float3 r1 = mk(eu * p01.x + fu * p11.x, eu * p01.y + fu * p11.y, eu * p01.z + fu * p11.z);
        const float ev = 1.0f - fv;
        r = mk(ev * r.x + fv * r1.x, ev * r.y + fv * r1.y, ev * r.z + fv * r1.z);
    }
    return r;
}

// FBm::doScalarLookUp (fbm.cpp:76-101): 1 - log2(footprint^2) / 2 octaves, clamped to [1, octaves],
// the fraction of the last one blended in; p[0] = 0 is plain Perlin noise (perlin.cpp:60-90)
__device__ inline float noise_texture(const DScene& S, const liar_texture& T, const TexPoint& q) {
    const uint8_t* tab = S.noise_tables + T.pixels;
    const int octaves = (int)T.p[0];
    if (octaves <= 0) return perlin_noise(tab, q.x);
    const float ideal = 1.0f - log2f(q.fp2) / 2.0f;  // +inf for a zero footprint
    const float real = fminf(fmaxf(ideal, 1.0f), (float)octaves);
    const int n = (int)floorf(real);
    float result = 0.0f, freq = 1.0f, weight = 1.0f;
    for (int k = 0; k < n; ++k) {
        result += weight * perlin_noise(tab, freq * q.x);
        freq *= 2.0f;
        weight *= T.p[1];
    }
    const float frac = real - (float)n;
    if (frac > 0.0f) result += frac * weight * perlin_noise(tab, freq * q.x);
    return result;
}

// Texture::lookUp of a texture tree (src/liar/textures/): transforms move (u, v) and its
// derivatives, boards pick a child or (anti-aliased CheckerBoard) blend both, images and noise are
// leaves, ABS / AFFINE apply to the value below them (abs.cpp:26-35; Product / Sum with constants,
// product.cpp:90-99, sum.cpp:90-105, look their input up as an illuminant and clamp as a
// reflectance), anything else is its spectrum. The operators waiting for values below them sit on a
// frame stack of at most kTexOps entries (the scene upload refuses trees with more on one path).
// Kept out of line, reading the scene from its device copy, so the shading kernels carry one call
// instead of the lookup's registers and frame.
constexpr int kTexOps = 8;
struct TexFrame {
    int op;        // LIAR_TEX_ABS, LIAR_TEX_AFFINE, or LIAR_TEX_CHECKER (a blend)
    float a, b;    // AFFINE: a v + b; CHECKER: the weight of child A in a
    bool refl;     // the caller's spectral type
    bool second;   // CHECKER: child A's value is in va, child B is being looked up
    float va;
    int tb;        // CHECKER: child B, looked up at q
    TexPoint q;
};
static __device__ __noinline__ float texture_eval(const DScene* __restrict__ G, int t, TexPoint q, float lam,
                                                  bool reflectant) {
    const DScene& S = *G;
    TexFrame fr[kTexOps];
    int n = 0;
    while (true) {
        // ---- down: from node t to a leaf value, pushing the operators met on the way
        float val = 0.0f;
        for (int steps = 0;; ++steps) {
            if (steps >= 64 || t < 0 || t >= S.n_tex) return 0.0f;
            const liar_texture T = S.texs[t];
            if (T.type == LIAR_TEX_CHECKER) {
                const float wa = checker_weight(T, q);
                if (wa >= 1.0f) {
                    t = T.a;
                } else if (wa <= 0.0f) {
                    t = T.b;
                } else {
                    // Spectral(wA A + (1 - wA) B, type) of the two looked up as illuminants
                    if (n == kTexOps) return 0.0f;
                    fr[n++] = TexFrame{LIAR_TEX_CHECKER, wa, 0.0f, reflectant, false, 0.0f, T.b, q};
                    reflectant = false;
                    t = T.a;
                }
            } else if (T.type == LIAR_TEX_GRID) {
                const float fu = q.u - floorf(q.u), fv = q.v - floorf(q.v);
                const bool on = fu < T.p[0] || fv < T.p[0] || fu > 1.0f - T.p[0] || fv > 1.0f - T.p[1];
                t = on ? T.a : T.b;
            } else if (T.type == LIAR_TEX_UV_TRANSFORM) {
                TexPoint m = q;
                m.u = T.p[0] * q.u + T.p[1] * q.v + T.p[2];
                m.v = T.p[3] * q.u + T.p[4] * q.v + T.p[5];
                m.du_i = T.p[0] * q.du_i + T.p[1] * q.dv_i;
                m.dv_i = T.p[3] * q.du_i + T.p[4] * q.dv_i;
                m.du_j = T.p[0] * q.du_j + T.p[1] * q.dv_j;
                m.dv_j = T.p[3] * q.du_j + T.p[4] * q.dv_j;
                q = m;
                t = T.a;
            } else if (T.type == LIAR_TEX_ABS || T.type == LIAR_TEX_AFFINE) {
                if (n == kTexOps) return 0.0f;
                fr[n++] = TexFrame{T.type, T.p[0], T.p[1], reflectant, false, 0.0f, -1, q};
                if (T.type == LIAR_TEX_AFFINE) reflectant = false;  // the input looked up as an illuminant
                t = T.a;
            } else if (T.type == LIAR_TEX_IMAGE) {
                // Image::doLookUp: Spectral::fromXYZ of the looked-up colour
                const float3 c = image_lookup(S, T, q);
                RecoveryBlend b;
                val = recovery_locate(S.rec, c.x, c.y, c.z, b) ? recovery_eval(S.rec, b, lam, reflectant) : 0.0f;
                break;
            } else if (T.type == LIAR_TEX_NOISE) {
                const float v = noise_texture(S, T, q);  // Spectral(value, type): min(value, 1) as a reflectance
                val = reflectant ? fminf(v, 1.0f) : v;
                break;
            } else {
                val = spec_eval(S, T.spectrum, lam, reflectant);
                break;
            }
        }
        // ---- up: apply the waiting operators; a blend whose first child is done looks up its second
        bool descend = false;
        while (n > 0 && !descend) {
            TexFrame& f = fr[n - 1];
            if (f.op == LIAR_TEX_ABS) {
                val = fabsf(val);
                --n;
            } else if (f.op == LIAR_TEX_AFFINE) {
                val = f.a * val + f.b;
                if (f.refl) val = fminf(val, 1.0f);
                --n;
            } else if (!f.second) {
                f.second = true;
                f.va = val;
                t = f.tb;
                q = f.q;
                reflectant = false;
                descend = true;
            } else {
                val = f.a * f.va + (1.0f - f.a) * val;
                if (f.refl) val = fminf(val, 1.0f);
                --n;
            }
        }
        if (!descend) return val;
    }
}

// a material parameter: its texture at the hit, else its constant spectrum
// (TEX false: a kernel instance for scenes without textures, which carries no lookup)
template <bool TEX>
__device__ __forceinline__ float param_eval(const DScene& S, const liar_material& M, int k, const HitContext& H,
                                            float lam, bool reflectant) {
    if (TEX && M.tex[k] >= 0)
        return texture_eval(S.self, M.tex[k], TexPoint{H.uv_u, H.uv_v, H.du_i, H.dv_i, H.du_j, H.dv_j, H.fp2, H.target},
                            lam, reflectant);
    return spec_eval(S, M.spec[k], lam, reflectant);
}

// Shader::bsdf at one wavelength
template <bool TEX = true>
__device__ inline Bsdf make_bsdf(const DScene& S, const liar_material& M, const HitContext& H, float lam) {
    Bsdf B;
    B.type = (uint32_t)M.type;
    B.mdf = M.mdf;
    B.ng = mk(dot(H.ng, H.u), dot(H.ng, H.v), dot(H.ng, H.N));
    B.r = B.t = 0.0f;
    B.eta = B.kappa = B.ior = B.eta_i = B.eta_t = 1.0f;
    B.au = sqr(fmaxf(M.rough_u, 1e-3f));
    B.av = sqr(fmaxf(M.rough_v, 1e-3f));
    switch (M.type) {
        case LIAR_MAT_LAMBERT:
            B.caps = CAP_REFL | CAP_DIFF;
            B.r = param_eval<TEX>(S, M, 0, H, lam, true);
            break;
        case LIAR_MAT_CONDUCTOR:
        case LIAR_MAT_COOK_TORRANCE:
            B.caps = M.type == LIAR_MAT_CONDUCTOR ? (CAP_REFL | CAP_SPEC) : (CAP_REFL | CAP_GLOSSY);
            B.eta = fmaxf(param_eval<TEX>(S, M, 0, H, lam, false), 1e-9f);
            B.kappa = fmaxf(param_eval<TEX>(S, M, 1, H, lam, false), 1e-9f);
            B.r = param_eval<TEX>(S, M, 2, H, lam, true);
            break;
        case LIAR_MAT_DIELECTRIC: {
            B.caps = CAP_REFL | CAP_TRANS | CAP_SPEC;
            const float ior1 = fmaxf(param_eval<TEX>(S, M, 1, H, lam, false), 1e-9f);
            const float ior2 = fmaxf(param_eval<TEX>(S, M, 0, H, lam, false), 1e-9f);
            B.ior = H.leaving ? ior2 / ior1 : ior1 / ior2;
            B.r = param_eval<TEX>(S, M, 2, H, lam, true);
            B.t = param_eval<TEX>(S, M, 3, H, lam, true);
            break;
        }
        case LIAR_MAT_WALTER: {
            B.caps = CAP_TRANS | CAP_GLOSSY;  // as constructed by Walter::Bsdf (walter.cpp:247)
            float ei = fmaxf(param_eval<TEX>(S, M, 1, H, lam, false), 1e-9f);
            float et = fmaxf(param_eval<TEX>(S, M, 0, H, lam, false), 1e-9f);
            if (H.leaving) {
                const float tmp = ei;
                ei = et;
                et = tmp;
            }
            B.eta_i = ei;
            B.eta_t = et;
            B.r = param_eval<TEX>(S, M, 2, H, lam, true);
            B.t = param_eval<TEX>(S, M, 3, H, lam, true);
            break;
        }
        case LIAR_MAT_MIRROR:
            B.caps = CAP_REFL | CAP_SPEC;
            B.r = param_eval<TEX>(S, M, 0, H, lam, true);
            break;
        default:
            B.caps = 0;
    }
    return B;
}

// PerspectiveCamera::doGenerateRay (cameras/perspective_camera.cpp:406-434) for the pixel and
// sample of key k: stratified jitter in the pixel, thin-lens when the lens radius and focus
// distance are set; the ray's limits scale the camera's near/far planes by 1 / cos(axis angle)
// PerspectiveCamera::doGenerateRay at screen point (sx, sy) and lens sample (lu, lv)
__device__ inline void camera_ray_at(const liar_camera& C, float sx, float sy, float lu, float lv, float3& pos,
                                     float3& dir, float& factor) {
    pos = mk(C.position[0], C.position[1], C.position[2]);
    dir = mk(C.direction[0], C.direction[1], C.direction[2]) + (sx - 0.5f) * mk(C.right[0], C.right[1], C.right[2]) +
          (sy - 0.5f) * mk(C.down[0], C.down[1], C.down[2]);
    dir = normal(dir);
    const float3 dn = mk(C.direction_normal[0], C.direction_normal[1], C.direction_normal[2]);
    factor = 1.0f / dot(dir, dn);
    if (C.lens_radius > 0.0f && C.focus_distance > 0.0f && C.focus_distance < 3.4e38f) {
        const float2 lens = concentric_disk(lu, lv);
        const float3 lp = pos + (C.lens_radius * lens.x) * mk(C.right_normal[0], C.right_normal[1], C.right_normal[2]) +
                          (C.lens_radius * lens.y) * mk(C.down_normal[0], C.down_normal[1], C.down_normal[2]);
        const float3 fp = pos + (factor * C.focus_distance) * dir;
        pos = lp;
        dir = normal(fp - lp);
        factor = 1.0f / dot(dir, dn);
    }
}

// screen and lens samples of key k
__device__ __forceinline__ void camera_samples(const SampleKey& k, int width, int height, float& sx, float& sy,
                                               float& lu, float& lv) {
    const uint32_t px = k.pixel % (uint32_t)width, py = k.pixel / (uint32_t)width;
    float jx, jy;
    sample_2d(k, DIM_SCREEN, jx, jy);
    sx = ((float)px + jx) / (float)width;
    sy = ((float)py + jy) / (float)height;
    lu = lv = 0.5f;
    sample_2d(k, DIM_LENS, lu, lv);
}

// PerspectiveCamera::doGenerateRay (cameras/perspective_camera.cpp:406-434) for the pixel and
// sample of key k: stratified jitter in the pixel, thin-lens when the lens radius and focus
// distance are set; the ray's limits scale the camera's near/far planes by 1 / cos(axis angle)
__device__ inline liar_ray camera_ray(const liar_camera& C, const SampleKey& k, int width, int height) {
    float sx, sy, lu, lv;
    camera_samples(k, width, height, sx, sy, lu, lv);
    float3 pos, dir;
    float factor;
    camera_ray_at(C, sx, sy, lu, lv, pos, dir, factor);
    return liar_ray{pos.x, pos.y, pos.z, fmaxf(kTol, factor * C.near_limit), dir.x, dir.y, dir.z, factor * C.far_limit};
}

// Camera::primaryRay's two differential rays (kernel/camera.cpp:53-60): the same lens sample at the
// screen point moved by one sample spacing along x and along y; RenderEngine spaces them
// 1 / (resolution sqrt(samples per pixel)) apart (render_engine.cpp:211-215)
__device__ inline void camera_differentials(const liar_camera& C, const SampleKey& k, int width, int height,
                                            float3& oi, float3& di, float3& oj, float3& dj) {
    float sx, sy, lu, lv, f;
    camera_samples(k, width, height, sx, sy, lu, lv);
    const float root = sqrtf((float)k.spp);
    const float dsx = 1.0f / ((float)width * root), dsy = 1.0f / ((float)height * root);
    camera_ray_at(C, sx + dsx, sy, lu, lv, oi, di, f);
    camera_ray_at(C, sx, sy + dsy, lu, lv, oj, dj, f);
}

// dPoint/du and dPoint/dv of a hit's surface parametrisation: a triangle's corner uvs (without
// them its barycentrics, so the edges), a sphere's spherical angles (sphere.cpp:150-172)
__device__ inline bool hit_dpduv(const DScene& S, uint32_t prim, float3 n_out, float3& dpdu, float3& dpdv) {
    if (prim >= S.n_tris) {
        const float r = S.spheres[prim - S.n_tris].w;
        constexpr float kPi = 3.14159265358979323846f;
        const float theta = acosf(fminf(fmaxf(n_out.z, -1.0f), 1.0f));
        const float st = sinf(theta);
        dpdu = (r * 2.0f * kPi) * mk(-n_out.y, n_out.x, 0.0f);
        if (st != 0.0f) {
            const float cs = n_out.z / st;
            dpdv = (r * kPi) * mk(cs * n_out.x, cs * n_out.y, -st);
        } else {
            const float phi = atan2f(n_out.y, n_out.x);
            dpdv = (r * kPi) * mk(cosf(phi), sinf(phi), 0.0f);
        }
        return true;
    }
    const uint32_t i0 = S.tri_idx[3 * prim], i1 = S.tri_idx[3 * prim + 1], i2 = S.tri_idx[3 * prim + 2];
    const float3 a = mk(S.verts[3 * i0], S.verts[3 * i0 + 1], S.verts[3 * i0 + 2]);
    const float3 e1 = mk(S.verts[3 * i1], S.verts[3 * i1 + 1], S.verts[3 * i1 + 2]) - a;
    const float3 e2 = mk(S.verts[3 * i2], S.verts[3 * i2 + 1], S.verts[3 * i2 + 2]) - a;
    if (!S.tri_uv) {
        dpdu = e1;
        dpdv = e2;
        return true;
    }
    const float* t = S.tri_uv + 6 * (size_t)prim;
    const float du1 = t[2] - t[0], dv1 = t[3] - t[1], du2 = t[4] - t[0], dv2 = t[5] - t[1];
    const float det = du1 * dv2 - dv1 * du2;
    if (det == 0.0f) return false;
    const float inv = 1.0f / det;
    dpdu = inv * (dv2 * e1 - dv1 * e2);
    dpdv = inv * (du1 * e2 - du2 * e1);
    return true;
}

// IntersectionContext::setScreenSpaceDifferentialsI (intersection_context.cpp:295-324) for both
// differential rays: each meets the tangent plane of the hit (shading normal, hit point); dPoint
// is the offset of that point, dUv solves dPoint = dPdU du + dPdV dv on the two axes other than the
// plane's major axis (Cramer's rule); a ray parallel to the plane, or a degenerate
// parametrisation, leaves a zero footprint
__device__ inline void hit_footprint(const DScene& S, HitContext& H, uint32_t prim, float3 oi, float3 di, float3 oj,
                                     float3 dj) {
    float3 n_out = H.N;
    if (prim >= S.n_tris) {
        const float4 sp = S.spheres[prim - S.n_tris];
        n_out = normal(H.target - mk(sp.x, sp.y, sp.z));
    }
    float3 dpdu, dpdv;
    if (!hit_dpduv(S, prim, n_out, dpdu, dpdv)) return;
    const float3 N = H.N, P = H.target;
    const float ax = fabsf(N.x), ay = fabsf(N.y), az = fabsf(N.z);
    const int major = ax >= ay ? (ax >= az ? 0 : 2) : (ay >= az ? 1 : 2);
    const int a = (major + 1) % 3, b = (major + 2) % 3;
    auto comp = [](float3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); };
    const float m00 = comp(dpdu, a), m01 = comp(dpdv, a), m10 = comp(dpdu, b), m11 = comp(dpdv, b);
    const float det = m00 * m11 - m01 * m10;
    float fp2 = 0.0f;
    for (int side = 0; side < 2; ++side) {
        const float3 o = side ? oj : oi, d = side ? dj : di;
        const float nd = dot(N, d);
        if (nd == 0.0f) continue;
        const float t = dot(N, P - o) / nd;
        if (!(t >= 0.0f)) continue;
        const float3 dp = (o + t * d) - P;
        fp2 = fmaxf(fp2, dot(dp, dp));
        if (det == 0.0f) continue;
        const float ra = comp(dp, a), rb = comp(dp, b);
        const float du = (ra * m11 - m01 * rb) / det, dv = (m00 * rb - ra * m10) / det;
        if (side) {
            H.du_j = du;
            H.dv_j = dv;
        } else {
            H.du_i = du;
            H.dv_i = dv;
        }
    }
    H.fp2 = fp2;
}

// the footprint of a camera hit: the camera's differential rays for key k (the camera vertex only;
// rays past it carry none, as the reference's DifferentialRay(BoundedRay) does)
__device__ inline void camera_footprint(const DScene& S, HitContext& H, uint32_t prim, const liar_camera& C,
                                        const SampleKey& k, int width, int height) {
    float3 oi, di, oj, dj;
    camera_differentials(C, k, width, height, oi, di, oj, dj);
    hit_footprint(S, H, prim, oi, di, oj, dj);
}

// ---- the film (output/raster.cpp:547-606, output/filter_triangle.cpp, output/filter_mitchell.cpp)

struct FilmSpec {
    float* film;         // width x height x 8 sums
    int width, height;
    int filter;          // liar_filter
    float param;         // triangle width / Mitchell B
    float max_lum;       // Raster.maxSampleLuminance, <= 0: none
};

// the filter settings of a render description, or nullptr when they are valid
__host__ inline const char* film_desc_error(const liar_render_desc& R) {
    if (R.filter != LIAR_FILTER_BOX && R.filter != LIAR_FILTER_TRIANGLE && R.filter != LIAR_FILTER_MITCHELL)
        return "unknown reconstruction filter";
    if (R.filter == LIAR_FILTER_TRIANGLE && !(R.filter_param >= 0.0f && R.filter_param <= 8.0f))
        return "triangle filter width must be in (0, 8] (0 selects 1)";
    if (R.filter == LIAR_FILTER_MITCHELL && !(R.filter_param >= -8.0f && R.filter_param <= 8.0f))
        return "Mitchell filter B out of range";
    if (!(R.max_sample_luminance >= 0.0f)) return "max_sample_luminance must be >= 0 (0: no clamp)";
    return nullptr;
}

__host__ inline FilmSpec film_spec(float* film, const liar_render_desc& R) {
    FilmSpec F;
    F.film = film;
    F.width = R.width;
    F.height = R.height;
    F.filter = R.filter;
    F.param = R.filter == LIAR_FILTER_TRIANGLE ? (R.filter_param > 0.0f ? R.filter_param : 1.0f)
                                               : (R.filter_param != 0.0f ? R.filter_param : 1.0f / 3.0f);
    F.max_lum = R.max_sample_luminance;
    return F;
}

// FilterMitchell::filterKernel (filter_mitchell.cpp:133-146), C = (1 - B) / 2
__device__ __forceinline__ float mitchell_kernel(float x, float B) {
    const float C = (1.0f - B) / 2.0f;
    x = fabsf(x);
    if (x < 1.0f)
        return ((12.0f - 9.0f * B - 6.0f * C) * (x * x * x) + (-18.0f + 12.0f * B + 6.0f * C) * (x * x) + (6.0f - 2.0f * B)) / 6.0f;
    if (x < 2.0f)
        return ((-B - 6.0f * C) * (x * x * x) + (6.0f * B + 30.0f * C) * (x * x) + (-12.0f * B - 48.0f * C) * x +
                (8.0f * B + 24.0f * C)) / 6.0f;
    return 0.0f;
}

__device__ __forceinline__ void film_add(float* f, float3 xyz, float alpha, float w) {
    const float wa = w * alpha;
    atomicAdd(f + 0, wa * xyz.x);
    atomicAdd(f + 1, wa * xyz.y);
    atomicAdd(f + 2, wa * xyz.z);
    atomicAdd(f + 3, wa);
    atomicAdd(f + 4, w * (xyz.x * xyz.x));
    atomicAdd(f + 5, w * (xyz.y * xyz.y));
    atomicAdd(f + 6, w * (xyz.z * xyz.z));
    atomicAdd(f + 7, w);
}

// One sample into the film. The box filter adds it to its own pixel with weight 1. The triangle
// and Mitchell filters spread it over the pixels within their radius with the weights the
// reference's filters give: the pixel at offset (i, j) gets k(dx + i) k(dy + j), with (dx, dy) the
// sample's offset from its pixel's centre (the reference adds the offset, so the footprint is
// mirrored about the pixel centre); pixels outside the image are dropped, as Raster drops them.
// A sample brighter than max_lum in Y is scaled down to it first.
__device__ inline void film_splat(const FilmSpec& F, const SampleKey& k, float3 xyz, float alpha) {
    if (F.max_lum > 0.0f && xyz.y > F.max_lum) {
        const float s = F.max_lum / xyz.y;
        xyz = mk(xyz.x * s, xyz.y * s, xyz.z * s);
    }
    if (F.filter == LIAR_FILTER_BOX) {
        film_add(F.film + 8 * (size_t)k.pixel, xyz, alpha, 1.0f);
        return;
    }
    const int px = (int)(k.pixel % (uint32_t)F.width), py = (int)(k.pixel / (uint32_t)F.width);
    float jx, jy;
    sample_2d(k, DIM_SCREEN, jx, jy);
    const float dx = jx - 0.5f, dy = jy - 0.5f;
    const bool mitchell = F.filter == LIAR_FILTER_MITCHELL;
    const int r = mitchell ? 2 : (int)ceilf(F.param);
    for (int j = -r; j <= r; ++j) {
        const int y = py + j;
        if (y < 0 || y >= F.height) continue;
        const float fy = mitchell ? mitchell_kernel(dy + (float)j, F.param) : fmaxf(0.0f, F.param - fabsf(dy + (float)j));
        for (int i = -r; i <= r; ++i) {
            const int x = px + i;
            if (x < 0 || x >= F.width) continue;
            const float fx = mitchell ? mitchell_kernel(dx + (float)i, F.param) : fmaxf(0.0f, F.param - fabsf(dx + (float)i));
            film_add(F.film + 8 * ((size_t)y * F.width + x), xyz, alpha, fx * fy);
        }
    }
}

}  // namespace rt
}  // namespace liar_gpu
