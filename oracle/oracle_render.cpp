// oracle_render.cpp -- CPU ORACLE (test infrastructure only) of the spectral path tracer.
//
// Loaded only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference leg;
// the product never calls it. A recursive restatement, in the reference's own structure and in
// single precision, of:
//   AdjointPhotonTracer::tracePhoton / shadeSurface / scatterSurface
//        (src/liar/tracers/adjoint_photon_tracer.cpp:84-292)
//   IntersectionContext flipTo / bsdfToLocal (src/liar/kernel/intersection_context.cpp:197-290)
//   Bsdf::evaluate / sample caps rules (src/liar/kernel/bsdf.cpp:52-98, bsdf.h:141-145)
//   Lambert, Conductor, CookTorrance, Dielectric, Walter, Mirror BSDFs and the GGX / Beckmann
//        distributions (src/liar/shaders/*.cpp, src/liar/kernel/microfacet.cpp)
//   LightArea / LightPoint / LightSky emission and sampling, LightContexts power CDF
//        (src/liar/scenery/light_*.cpp, src/liar/kernel/light_context.cpp:272-333)
//   Observer sample / sensitivity and Spectral::xyz in Single mode
//        (src/liar/kernel/observer.cpp:57-171,283-317, src/liar/kernel/spectral.cpp:178-220)
//   Sampled / BlackBody / Cauchy spectra (src/liar/spectra/*.cpp)
// Scene intersection uses the oracle's own tree (oracle_trace.cpp) with the same hit rule.
// The sample values come from the same stratified hash sampler definition as the product, so
// both consume identical random numbers; results still differ where the libm
// transcendentals (sin, cos, exp, log, tan, atan) round differently on the two machines.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "../include/liar_gpu.h"

extern "C" int oracle_tri_intersect(const float* o, const float* d, const float* a, const float* b, const float* c,
                                    float* t_out, float* u_out, float* v_out);
extern "C" void* oracle_tree_build(const float* V, uint64_t nv, const uint32_t* T, uint64_t nt);
extern "C" void oracle_tree_free(void* tree);
extern "C" void oracle_tree_set_spheres(void* tree, const float* spheres, uint64_t n, uint64_t n_tris);

namespace oracle_internal {
struct Ray {
    float ox, oy, oz, tmin, dx, dy, dz, tmax;
};
struct Hit {
    int32_t prim;
    float t;
};
Hit tree_closest(void* tree, const Ray& r);
bool tree_any(void* tree, const Ray& r);
}  // namespace oracle_internal

namespace {

using oracle_internal::Hit;
using oracle_internal::Ray;

// ---- scene description (same memory layout as the library's C ABI structs)
struct Spectrum {
    int32_t type, offset, count;
    float p[3];
};
struct Material {
    int32_t type, mdf;
    int32_t spec[4];
    int32_t emission;
    float rough_u, rough_v;
    int32_t samples;
    int32_t tex[4];
};
struct Texture {
    int32_t type, a, b, spectrum;
    float p[6];
    int64_t pixels;
};
struct Light {
    int32_t type, spectrum, object, double_sided;
    int32_t first_tri, n_tris;
    float pos[3], u[3], v[3];
    float power;
    int32_t emission_samples;
};
struct Camera {
    float position[3], direction[3], right[3], down[3];
    float direction_normal[3], right_normal[3], down_normal[3];
    float lens_radius, focus_distance, near_limit, far_limit;
};
struct SceneIn {
    const float* vertices; uint64_t n_vertices;
    const uint32_t* triangles; uint64_t n_triangles;
    const int32_t* triangle_object;
    const float* normals; uint64_t n_normals;
    const int32_t* triangle_normals;
    const int32_t* object_material; const int32_t* object_light; uint64_t n_objects;
    const Material* materials; uint64_t n_materials;
    const Spectrum* spectra; uint64_t n_spectra;
    const float* pool; uint64_t pool_size;
    const Light* lights; uint64_t n_lights;
    const float* observer; uint64_t n_observer;
    float scene_radius;
    const Texture* textures; uint64_t n_textures;
    const float* triangle_uvs;
    const float* texture_pixels; uint64_t n_texture_pixels;
    const uint8_t* noise_tables; uint64_t n_noise_tables;
    const float* spheres; uint64_t n_spheres; const int32_t* sphere_object;
};
struct RenderIn {
    Camera camera;
    int32_t width, height, spp, tracer, max_ray_generation, max_depth;
    uint64_t seed;
    int32_t first_sample, wave_paths;
    int32_t secondary_light_samples, trace_glossy;
    int32_t filter;
    float filter_param, max_sample_luminance;
    // PhotonMapper settings (liar_photon_mapper_desc); the oracle takes its maps as PmIn instead
    uint64_t pm_max_photons, pm_global_map_size;
    float pm_radius[2], pm_tolerance[2];
    int32_t pm_size[2], pm_ray_trace_direct, pm_visualize;
    int32_t pm_final_gather_rays, pm_secondary_gather_rays;
    float pm_ratio_precomputed_irradiance;
    float pm_caustics_quality;
    int32_t sampler;  // LIAR_SAMPLER_* bits
};

// the mirrors above have the C ABI's layout
static_assert(sizeof(Spectrum) == sizeof(liar_spectrum) && sizeof(Material) == sizeof(liar_material) &&
                  sizeof(Texture) == sizeof(liar_texture) && sizeof(Light) == sizeof(liar_light) &&
                  sizeof(Camera) == sizeof(liar_camera) && sizeof(SceneIn) == sizeof(liar_scene_desc) &&
                  sizeof(RenderIn) == sizeof(liar_render_desc),
              "oracle mirrors out of step with include/liar_gpu.h");
static_assert(offsetof(Material, tex) == offsetof(liar_material, tex) &&
                  offsetof(SceneIn, triangle_uvs) == offsetof(liar_scene_desc, triangle_uvs) &&
                  offsetof(RenderIn, pm_max_photons) == offsetof(liar_render_desc, photon_mapper) &&
                  offsetof(RenderIn, filter) == offsetof(liar_render_desc, filter) &&
                  offsetof(RenderIn, sampler) == offsetof(liar_render_desc, sampler) &&
                  offsetof(Texture, pixels) == offsetof(liar_texture, pixels) &&
                  offsetof(SceneIn, texture_pixels) == offsetof(liar_scene_desc, texture_pixels) &&
                  offsetof(SceneIn, noise_tables) == offsetof(liar_scene_desc, noise_tables) &&
                  offsetof(SceneIn, sphere_object) == offsetof(liar_scene_desc, sphere_object),
              "oracle mirrors out of step with include/liar_gpu.h");

// The photon maps of a PhotonMapper render (photon_mapper.cpp:798-835) as the oracle gets them:
// photons in buffer order, powers XYZ already scaled, each power's recovery blend (three sample
// indices, -1 = none, and weights); the standard recovery table for colours located here.
struct PmIn {
    const float* position[2];
    const float* omega_in[2];
    const float* power[2];
    const int32_t* blend_idx[2];
    const float* blend_w[2];
    uint64_t n[2];
    float radius[2];
    int32_t k[2];
    int32_t visualize, ray_direct;
    const float* rec_wavelengths;
    const float* rec_spectra;
    const float* rec_points;   // (n_samples + 4) x 2
    const int32_t* rec_tris;
    int32_t rec_nw, rec_ns, rec_nt;
    // final gathering: rays per high-quality diffuse vertex (0: none), secondary rays, and the
    // irradiance map (points, normals, blends of the irradiance, squared radii)
    int32_t fg_rays, fg_secondary;
    const float* irr_position;
    const float* irr_normal;
    const int32_t* irr_blend_idx;
    const float* irr_blend_w;
    const float* irr_r2;
    uint64_t n_irr;
};

enum { SP_CONST = 0, SP_SAMPLED = 1, SP_BB = 2, SP_CAUCHY = 3 };
enum { M_NONE = 0, M_LAMBERT = 1, M_CONDUCTOR = 2, M_CT = 3, M_DIELECTRIC = 4, M_WALTER = 5, M_MIRROR = 6 };
enum { L_PARA = 0, L_MESH = 1, L_POINT = 2, L_SKY = 3 };
enum { C_REFL = 0x2, C_TRANS = 0x4, C_DIFF = 0x10, C_SPEC = 0x20, C_GLOSSY = 0x40, C_ALL = 0xff };
const float PI = 3.14159265358979323846f;
const float TOL = 1e-6f;

// ---- vectors
struct V {
    float x, y, z;
};
V operator+(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V operator-(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V operator-(V a) { return {-a.x, -a.y, -a.z}; }
V operator*(float s, V a) { return {s * a.x, s * a.y, s * a.z}; }
float dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V cross(V a, V b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
float len(V a) { return std::sqrt(dot(a, a)); }
V unit(V a) { return (1.0f / len(a)) * a; }
float sq(float x) { return x * x; }
V reflect(V h, V v) { return (2.0f * dot(h, v)) * h - v; }  // Lass Vector3D::reflect

// ---- sampler (the same definition as the library's sampler)
uint64_t mix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
float unitf(uint64_t h) { return (float)(uint32_t)(h >> 40) * (1.0f / 16777216.0f); }
uint32_t permute(uint32_t i, uint32_t n, uint64_t key) {
    if (n <= 1) return 0;
    uint32_t bits = 0;
    while ((1u << bits) < n) ++bits;
    if (bits & 1u) ++bits;
    const uint32_t half = bits / 2, mask = (1u << half) - 1u;
    do {
        uint32_t l = i >> half, r = i & mask;
        for (uint32_t k = 0; k < 4; ++k) {
            const uint32_t f = (uint32_t)mix64(key + 0x632be59bd9b4e019ull * (k + 1) + r) & mask;
            const uint32_t nl = r;
            r = l ^ f;
            l = nl;
        }
        i = (l << half) | r;
    } while (i >= n);
    return i;
}
// mode bits: LIAR_SAMPLER_LATIN_HYPERCUBE (screen and lens axes stratified one by one, the
// LatinHypercube, samplers/latin_hypercube.cpp) and LIAR_SAMPLER_NOT_JITTERED (stratum centres,
// samplers/stratifier.h:90); without them the Stratifier's 2D grid of screen and lens strata
// (samplers/stratifier.cpp:163-180)
struct Sampler {
    uint64_t seed;
    uint32_t pixel, sample, spp;
    uint32_t mode = 0;
    uint64_t hash(uint32_t dim) const { return mix64(seed ^ mix64(((uint64_t)pixel << 32) | (uint64_t)dim)); }
    float jitter(uint64_t hd) const { return unitf(mix64(hd + 0xd1b54a32d192ed03ull * ((uint64_t)sample + 1))); }
    float get(uint32_t dim, bool strat) const {
        const uint64_t hd = hash(dim);
        if (!strat) return jitter(hd);
        const float jit = (mode & LIAR_SAMPLER_NOT_JITTERED) ? 0.5f : jitter(hd);
        if (spp <= 1) return jit;
        const uint32_t s = permute(sample, spp, hd);
        const float u = ((float)s + jit) / (float)spp;
        return u < 1.0f ? u : 0.99999994f;
    }
    void get2(uint32_t dim, float& x, float& y) const {
        uint32_t n = 0;
        while ((n + 1) * (n + 1) <= spp) ++n;
        if ((mode & LIAR_SAMPLER_LATIN_HYPERCUBE) || spp <= 1 || n * n != spp) {
            x = get(dim, true);
            y = get(dim + 1, true);
            return;
        }
        const uint64_t hx = hash(dim), hy = hash(dim + 1);
        const uint32_t s = permute(sample, spp, hx);
        const bool jit = !(mode & LIAR_SAMPLER_NOT_JITTERED);
        const float jx = jit ? jitter(hx) : 0.5f, jy = jit ? jitter(hy) : 0.5f;
        const float u = ((float)(s % n) + jx) / (float)n, v = ((float)(s / n) + jy) / (float)n;
        x = u < 1.0f ? u : 0.99999994f;
        y = v < 1.0f ? v : 0.99999994f;
    }
};
const uint32_t D_SCREEN = 0, D_LENS = 2, D_LAMBDA = 4, D_GEN0 = 8, D_PER_GEN = 8;
const uint32_t O_STRAT = 0, O_BSDF = 1, O_COMP = 3, O_LCHOICE = 4, O_LIGHT = 5, O_RR = 7;

// ---- scene
// a recovery table (RecoveryMengSimon, recovery_meng_simon.cpp:93-310): spectra at chromaticity
// points, the triangulation of the points and the four box corners that follow them
struct RecView {
    const float* wavelengths = nullptr;
    const float* spectra = nullptr;
    const float* points = nullptr;   // (ns + 4) x 2
    const int32_t* tris = nullptr;
    int nw = 0, ns = 0, nt = 0;
};

struct Scene {
    SceneIn in;
    RecView rec;                     // for image textures (Spectral::fromXYZ)
    std::vector<float> rec_w, rec_s, rec_p;
    std::vector<int32_t> rec_t;
    void* tree = nullptr;
    std::vector<float> spec_max, light_cdf, light_area, tri_cdf;
    std::vector<float> ow, oxyz, odxyz, ocdf;
    int sky = -1;
    float sky_distance = 1e3f;
};

float planck(float w, float T) {
    const float h = 6.626070040e-34f, c = 299792458.0f, kb = 1.3806488e-23f;
    const float c1 = 2 * h * c * c, c2 = h * c / kb;
    const float w5 = sq(sq(w)) * w;
    return c1 / (w5 * std::expm1(c2 / (w * T)));
}

float spectrum(const Scene& S, int idx, float w, bool reflectant) {
    if (idx < 0) return 0.0f;
    const Spectrum& sp = S.in.spectra[idx];
    float v;
    if (sp.type == SP_SAMPLED) {
        const float* ws = S.in.pool + sp.offset;
        const float* vs = ws + sp.count;
        const float* it = std::upper_bound(ws, ws + sp.count, w);
        if (it == ws || it == ws + sp.count) return 0.0f;
        const int k = (int)(it - ws);
        const float t = (w - ws[k - 1]) / (ws[k] - ws[k - 1]);
        v = vs[k - 1] + t * (vs[k] - vs[k - 1]);
        if (reflectant && S.spec_max[idx] > 1.0f) return v / S.spec_max[idx];
        return v;
    } else if (sp.type == SP_BB) {
        const float T = sp.p[0];
        v = sp.p[1] * (1.0f / planck(2.897771955e-3f / T, T)) * planck(w, T);
    } else if (sp.type == SP_CAUCHY) {
        const float wu = w * 1e6f;
        v = sp.p[0] + sp.p[1] / sq(wu);
    } else {
        v = sp.p[0];
    }
    return reflectant ? std::min(v, 1.0f) : v;
}

float observer_sample(const Scene& S, float u, float& pdf) {
    const int n = (int)S.ow.size();
    const auto it = std::upper_bound(S.ocdf.begin(), S.ocdf.end(), u);
    if (it == S.ocdf.begin() || it == S.ocdf.end()) {
        pdf = 0;
        return it == S.ocdf.begin() ? S.ow[0] : S.ow[n - 1];
    }
    const int k = (int)(it - S.ocdf.begin());
    const float c1 = S.ocdf[k - 1], c2 = S.ocdf[k], dc = c2 - c1;
    const float x = (u - c1) / dc;
    pdf = dc / (S.ow[k] - S.ow[k - 1]);
    return S.ow[k - 1] + x * (S.ow[k] - S.ow[k - 1]);
}
V observer_sensitivity(const Scene& S, float w) {
    const auto it = std::upper_bound(S.ow.begin(), S.ow.end(), w);
    if (it == S.ow.begin() || it == S.ow.end()) return {0, 0, 0};
    const int k = (int)(it - S.ow.begin()) - 1;
    const float dw = w - S.ow[k];
    return {S.oxyz[3 * k] + S.odxyz[3 * k] * dw, S.oxyz[3 * k + 1] + S.odxyz[3 * k + 1] * dw,
            S.oxyz[3 * k + 2] + S.odxyz[3 * k + 2] * dw};
}

// ---- warps restated from their published methods
void concentric(float u1, float u2, float& x, float& y) {
    const float a = 2 * u1 - 1, b = 2 * u2 - 1;
    if (a == 0 && b == 0) {
        x = y = 0;
        return;
    }
    float r, phi;
    if (std::fabs(a) > std::fabs(b)) {
        r = a;
        phi = (PI / 4) * (b / a);
    } else {
        r = b;
        phi = (PI / 2) - (PI / 4) * (a / b);
    }
    x = r * std::cos(phi);
    y = r * std::sin(phi);
}
V cosine_hemisphere(float u1, float u2, float& pdf) {
    float x, y;
    concentric(u1, u2, x, y);
    const float z = std::sqrt(std::max(0.0f, 1 - x * x - y * y));
    pdf = z / PI;
    return {x, y, z};
}
V uniform_sphere(float u1, float u2, float& pdf) {
    const float z = 1 - 2 * u2;
    const float r = std::sqrt(std::max(0.0f, 1 - z * z));
    const float phi = 2 * PI * u1;
    pdf = 1 / (4 * PI);
    return {r * std::cos(phi), r * std::sin(phi), z};
}

// ---- BSDF (in the shading frame)
struct Bsdf {
    int type, mdf;
    uint32_t caps;
    V ng;
    float r, t, eta, kappa, ior, etaI, etaT, au, av;
};
struct Out {
    V wo;
    float value, pdf;
    explicit operator bool() const { return pdf > 0 && value != 0; }
};
bool has(uint32_t c, uint32_t w) { return (c & w) == w; }
bool compatible(uint32_t c, uint32_t a) {
    const uint32_t o = c & a;
    return (o & 0xf) > 0 && (o & 0xf0) > 0;
}

float sample_phi(float s, float au, float av) {
    if (au == av) return 2 * PI * s;
    const float phi = std::atan(av / au * std::tan(2 * PI * s));
    if (s <= 0.25f) return phi;
    if (s < 0.75f) return phi + PI;
    return phi + 2 * PI;
}
float D(int mdf, V h, float au, float av, float& pdfH) {
    if (mdf == 1) {  // Trowbridge-Reitz (GGX), microfacet_trowbridge_reitz.cpp:47-60
        const float d = 1.0f / (PI * au * av * sq(sq(h.x / au) + sq(h.y / av) + sq(h.z)));
        pdfH = d * h.z;
        return d;
    }
    const float c2 = sq(h.z);  // Beckmann, microfacet_beckmann.cpp:53-74
    if (c2 == 0) {
        pdfH = 0;
        return 0;
    }
    const float d = std::exp(-(sq(h.x / au) + sq(h.y / av)) / c2) / (PI * au * av * sq(c2));
    pdfH = d * h.z;
    return d;
}
V sample_h(int mdf, float sx, float sy, float au, float av) {
    if (mdf == 1) {
        const float phi = sample_phi(sx, au, av);
        const float s = std::sqrt(sy / (1 - sy));
        return unit({s * au * std::cos(phi), s * av * std::sin(phi), 1});
    }
    const float s = std::log(1 - sx);
    float cp, sp, t2;
    if (au == av) {
        const float phi = 2 * PI * sy;
        cp = std::cos(phi);
        sp = std::sin(phi);
        t2 = -s * sq(au);
    } else {
        const float phi = sample_phi(sx, au, av);
        cp = std::cos(phi);
        sp = std::sin(phi);
        t2 = -s / (sq(cp / au) + sq(sp / av));
    }
    const float c2 = 1 / (1 + t2);
    return {cp * std::sqrt(std::max(1 - c2, 0.0f)), sp * std::sqrt(std::max(1 - c2, 0.0f)), std::sqrt(c2)};
}
float lambda_(int mdf, V w, float au, float av) {
    if (mdf == 1) return (std::sqrt(1 + (sq(w.x * au) + sq(w.y * av)) / sq(w.z)) - 1) / 2;
    const float a2 = sq(w.z) / (sq(w.x * au) + sq(w.y * av));
    const float a = std::sqrt(a2);
    return a < 1.6f ? (3.535f * a + 2.181f * a2) / (1 + 2.276f * a + 2.577f * a2) : 1;
}
float G1(int mdf, V w, V h, float au, float av) {
    if (dot(w, h) * w.z <= 0) return 0;
    return 1 / (1 + lambda_(mdf, w, au, av));
}
float fresnel_cond(float eta, float kappa, float cosI) {
    const float c2 = sq(cosI), a = sq(eta) + sq(kappa), b = 2 * cosI * eta;
    const float aO = a + c2, aP = a * c2 + 1;
    return ((aO - b) / (aO + b) + (aP - b) / (aP + b)) / 2;
}
float fresnel_walter(float ior, V wi, V h) {
    const float cI = std::fabs(dot(wi, h));
    const float s2 = sq(ior) * (1 - sq(cI));
    const float cT = std::sqrt(std::max(1 - s2, 0.0f));
    const float rO = (ior * cI - cT) / (ior * cI + cT), rP = (cI - ior * cT) / (cI + ior * cT);
    return std::min((sq(rO) + sq(rP)) / 2, 1.0f);
}
float walter_pr(const Bsdf& b, float rF, uint32_t al) {
    const float pr = has(al, C_REFL | C_GLOSSY) ? std::fabs(b.r) * rF : 0;
    const float pt = has(al, C_TRANS | C_GLOSSY) ? std::fabs(b.t) * (1 - rF) : 0;
    if (pr + pt == 0) return -1;
    return pr / (pr + pt);
}

Out do_evaluate(const Bsdf& b, V wi, V wo, uint32_t al) {
    Out o{{0, 0, 0}, 0, 0};
    if (b.type == M_LAMBERT) {
        const float c = std::fabs(wo.z);
        if (c <= 0) return o;
        return {wo, b.r / PI, c / PI};
    }
    if (b.type == M_CT) {
        if (wo.z <= 0) return o;
        const V h = unit(wi + wo);
        float pdfH;
        const float d = D(b.mdf, h, b.au, b.av, pdfH);
        const float dh = std::fabs(dot(wi, h));
        const float g = std::min(1.0f, std::min(2 * h.z * wi.z / dh, 2 * h.z * wo.z / dh));
        const float pdf = pdfH / (4 * dot(wi, h));
        float v = b.r * (d * g / (4 * wi.z * wo.z));
        v *= fresnel_cond(b.eta, b.kappa, std::fabs(dot(wi, h)));
        return {wo, v, pdf};
    }
    if (b.type == M_WALTER) {
        if (wo.z > 0) {
            const V h = unit(wi + wo);
            const float rF = fresnel_walter(b.etaI / b.etaT, wi, h);
            const float pR = walter_pr(b, rF, al);
            if (pR < 0) return o;
            float pdfH;
            const float d = D(b.mdf, h, b.au, b.av, pdfH);
            const float g = G1(b.mdf, wi, h, b.au, b.av) * G1(b.mdf, wo, h, b.au, b.av);
            const float dh = 1 / (4 * dot(wi, h));
            return {wo, b.r * (rF * d * g / (4 * wi.z * wo.z)), pR * pdfH * dh};
        } else if (wo.z < 0) {
            const V h = unit(-(b.etaI * wi) - b.etaT * wo);
            if (h.z <= 0) return o;
            const float cI = std::fabs(dot(wi, h)), cT = std::fabs(dot(wo, h));
            const float rF = fresnel_walter(b.etaI / b.etaT, wi, h);
            const float pR = walter_pr(b, rF, al);
            if (pR < 0) return o;
            float pdfH;
            const float d = D(b.mdf, h, b.au, b.av, pdfH);
            const float g = G1(b.mdf, wi, h, b.au, b.av) * G1(b.mdf, wo, h, b.au, b.av);
            const float dh = sq(b.etaT) * cT / sq(b.etaI * cI + b.etaT * cT);
            return {wo, b.t * (((1 - rF) * d * g * (cI * dh)) / std::fabs(wi.z * wo.z)), (1 - pR) * pdfH * dh};
        }
    }
    return o;
}
Out evaluate(const Bsdf& b, V wi, V wo, uint32_t al) {
    if (wo.z == 0) return {wo, 0, 0};
    const bool refl = (dot(wi, b.ng) > 0) == (dot(wo, b.ng) > 0);
    al &= ~(refl ? (uint32_t)C_TRANS : (uint32_t)C_REFL);
    if (!compatible(b.caps, al)) return {wo, 0, 0};
    return do_evaluate(b, wi, wo, al);
}
Out sample(const Bsdf& b, V wi, float sx, float sy, float comp, uint32_t al) {
    Out o{{0, 0, 0}, 0, 0};
    if (!compatible(b.caps, al)) return o;
    switch (b.type) {
        case M_LAMBERT: {
            float pdf;
            const V wo = cosine_hemisphere(sx, sy, pdf);
            return {wo, b.r / PI, pdf};
        }
        case M_CONDUCTOR:
            return {{-wi.x, -wi.y, wi.z}, b.r * fresnel_cond(b.eta, b.kappa, wi.z) / wi.z, 1};
        case M_MIRROR:
            return {{-wi.x, -wi.y, wi.z}, b.r, wi.z};
        case M_CT: {
            const V h = sample_h(b.mdf, sx, sy, b.au, b.av);
            const V wo = reflect(h, wi);
            if (wo.z <= 0) return o;
            return do_evaluate(b, wi, wo, al);
        }
        case M_DIELECTRIC: {
            const float cI = wi.z;
            if (cI <= 0) return o;
            const float ior = b.ior;
            const float s2 = sq(ior) * (1 - sq(cI));
            const float cT = std::sqrt(std::max(1 - s2, 0.0f));
            const float rO = (ior * cI - cT) / (ior * cI + cT), rP = (cI - ior * cT) / (cI + ior * cT);
            const float rF = (sq(rO) + sq(rP)) / 2;
            const float pr = has(al, C_REFL | C_SPEC) ? std::fabs(b.r) * rF : 0;
            const float pt = has(al, C_TRANS | C_SPEC) ? std::fabs(b.t) * (1 - rF) : 0;
            if (pr + pt == 0) return o;
            const float probR = pr / (pr + pt);
            if (comp < probR) return {{-wi.x, -wi.y, wi.z}, b.r * rF / cI, probR};
            return {{-ior * wi.x, -ior * wi.y, -cT}, b.t * (1 - rF) / cT, 1 - probR};
        }
        case M_WALTER: {
            const V h = sample_h(b.mdf, sx, sy, b.au, b.av);
            float pdfH;
            const float d = D(b.mdf, h, b.au, b.av, pdfH);
            const float rF = fresnel_walter(b.etaI / b.etaT, wi, h);
            const float pR = walter_pr(b, rF, al);
            if (pR < 0) return o;
            if (comp < pR) {
                const V wo = reflect(h, wi);
                if (wo.z <= 0) return o;
                const float g = G1(b.mdf, wi, h, b.au, b.av) * G1(b.mdf, wo, h, b.au, b.av);
                const float dh = 1 / (4 * dot(wo, h));
                return {wo, b.r * (rF * d * g / (4 * wi.z * wo.z)), pR * pdfH * dh};
            }
            const float eta = b.etaI / b.etaT;
            const float cI = std::fabs(dot(wi, h));
            const float s2 = sq(eta) * (1 - sq(cI));
            const float cT = std::sqrt(std::max(1 - s2, 0.0f));
            const V wo = unit((-eta) * wi + (eta * cI - cT) * h);
            if (wo.z >= 0) return o;
            const float g = G1(b.mdf, wi, h, b.au, b.av) * G1(b.mdf, wo, h, b.au, b.av);
            const float dh = sq(b.etaT) * cT / sq(b.etaI * cI + b.etaT * cT);
            return {wo, b.t * (((1 - rF) * d * g * (cI * dh)) / std::fabs(wi.z * wo.z)), (1 - pR) * pdfH * dh};
        }
    }
    return o;
}

// ---- lights
float light_pdf_choice(const Scene& S, int k) { return k > 0 ? S.light_cdf[k] - S.light_cdf[k - 1] : S.light_cdf[0]; }

bool para_hit(const Light& L, V o, V d, float tmin, float& t) {
    const V p{L.pos[0], L.pos[1], L.pos[2]}, u{L.u[0], L.u[1], L.u[2]}, v{L.v[0], L.v[1], L.v[2]};
    const V n = cross(u, v);
    const float den = dot(n, d);
    if (den == 0) return false;
    const float th = dot(n, p - o) / den;
    if (!(th > tmin)) return false;
    const V x = o + th * d - p;
    const float uu = dot(u, u), uv = dot(u, v), vv = dot(v, v), xu = dot(x, u), xv = dot(x, v);
    const float det = uu * vv - uv * uv;
    const float a = (xu * vv - xv * uv) / det, b = (xv * uu - xu * uv) / det;
    if (a < 0 || a > 1 || b < 0 || b > 1) return false;
    t = th;
    return true;
}

// SceneLight::emission(ray): radiance and solid-angle pdf of the direction
float light_emission_pdf(const Scene& S, int li, V o, V d) {
    const Light& L = S.in.lights[li];
    if (L.type == L_PARA) {
        float t;
        if (!para_hit(L, o, d, TOL, t)) return 0;
        const V n = unit(cross({L.u[0], L.u[1], L.u[2]}, {L.v[0], L.v[1], L.v[2]}));
        return sq(t) / std::fabs(S.light_area[li] * dot(d, n));
    }
    if (L.type == L_MESH) {
        float tb = INFINITY;
        int best = -1;
        for (int k = 0; k < L.n_tris; ++k) {
            const uint32_t* tr = S.in.triangles + 3 * (size_t)(L.first_tri + k);
            const float oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
            float t, u, v;
            if (oracle_tri_intersect(oo, dd, S.in.vertices + 3 * tr[0], S.in.vertices + 3 * tr[1],
                                     S.in.vertices + 3 * tr[2], &t, &u, &v) && t > TOL && t < tb) {
                tb = t;
                best = L.first_tri + k;
            }
        }
        if (best < 0) return 0;
        const uint32_t* tr = S.in.triangles + 3 * (size_t)best;
        const float* a = S.in.vertices + 3 * tr[0];
        const float* b = S.in.vertices + 3 * tr[1];
        const float* c = S.in.vertices + 3 * tr[2];
        const V n = unit(cross({b[0] - a[0], b[1] - a[1], b[2] - a[2]}, {c[0] - a[0], c[1] - a[1], c[2] - a[2]}));
        return sq(tb) / std::fabs(S.light_area[li] * dot(d, n));
    }
    if (L.type == L_SKY) return 1 / (4 * PI);
    return 0;
}

struct LS {
    V dir;
    float pdf;
};
LS light_sample(const Scene& S, int li, V target, float sx, float sy) {
    const Light& L = S.in.lights[li];
    if (L.type == L_PARA || L.type == L_MESH) {
        V p, n;
        float pdf;
        if (L.type == L_PARA) {
            const V u{L.u[0], L.u[1], L.u[2]}, v{L.v[0], L.v[1], L.v[2]};
            p = V{L.pos[0], L.pos[1], L.pos[2]} + sx * u + sy * v;
            n = unit(cross(u, v));
            pdf = 1 / S.light_area[li];
        } else {
            const float* cdf = S.tri_cdf.data() + L.first_tri;
            int ii = (int)(std::lower_bound(cdf, cdf + L.n_tris, sx) - cdf);
            ii = std::min(ii, L.n_tris - 1);
            const float i0 = ii > 0 ? cdf[ii - 1] : 0.0f;
            const float tp = cdf[ii] - i0;
            const float di = (sx - i0) / tp;
            const uint32_t* tr = S.in.triangles + 3 * (size_t)(L.first_tri + ii);
            const float* a = S.in.vertices + 3 * tr[0];
            const float* b = S.in.vertices + 3 * tr[1];
            const float* c = S.in.vertices + 3 * tr[2];
            const V A{a[0], a[1], a[2]}, e1{b[0] - a[0], b[1] - a[1], b[2] - a[2]}, e2{c[0] - a[0], c[1] - a[1], c[2] - a[2]};
            const V nn = cross(e1, e2);
            const float s = std::sqrt(di);
            const float nl = len(nn);
            n = (1 / nl) * nn;
            pdf = tp / (nl / 2);
            p = A + (1 - s) * e1 + (s * sy) * e2;
        }
        V to = p - target;
        const float d2 = dot(to, to);
        to = (1 / std::sqrt(d2)) * to;
        pdf *= d2 / std::fabs(dot(n, to));
        V tl = p - target;
        tl = (1 / len(tl)) * tl;
        if (!L.double_sided && dot(n, tl) > 0) return {tl, 0};
        return {tl, pdf};
    }
    if (L.type == L_POINT) {
        V tl = V{L.pos[0], L.pos[1], L.pos[2]} - target;
        tl = (1 / len(tl)) * tl;
        return {tl, 1};
    }
    if (L.type == L_SKY) {
        float pdf;
        const V d = uniform_sphere(sx, sy, pdf);
        return {d, pdf};
    }
    return {{0, 0, 1}, 0};
}

float power_heuristic(float a, float b) { return sq(a) / (sq(a) + sq(b)); }

struct Path {
    const Scene* S;
    const RenderIn* R;
    Sampler smp;
    float lam;
    float alpha = 0;
};

float trace_photon(Path& P, V o, V d, float tmin, float tmax, int gen);

// IntersectionContext of a hit (intersection_context.cpp:55-290): point, flipped normals, frame
struct Ctx {
    V target, ng, N, u, v;
    bool leaving;
    int obj, light, mi;
    float uv_u, uv_v;
    // the screen-space footprint (dUv_dI, dUv_dJ, max |dPoint|^2): zero without ray differentials
    float du_i = 0, dv_i = 0, du_j = 0, dv_j = 0, fp2 = 0;
};

// IntersectionContext::uv of a triangle hit (TriangleMesh::doLocalContext, triangle_mesh.cpp:334-356):
// the corners' (u, v) interpolated at the barycentrics, or the barycentrics themselves
void hit_uv(const Scene& S, uint32_t prim, float bu, float bv, float& u, float& v) {
    if (!S.in.triangle_uvs) {
        u = bu;
        v = bv;
        return;
    }
    const float* t = S.in.triangle_uvs + 6 * (size_t)prim;
    const float w0 = 1 - bu - bv;
    u = w0 * t[0] + bu * t[2] + bv * t[4];
    v = w0 * t[1] + bu * t[3] + bv * t[5];
}

float frac(float x) { return x - std::floor(x); }

// RecoveryMengSimon::Impl::recover by a search of every triangle: blend of XYZ (three sample
// indices, -1 for a box corner, and weights scaled to X + Y + Z), false when there is none
bool rec_locate(const RecView& R, float X, float Y, float Z, int32_t idx[3], float w[3]) {
    const float s = X + Y + Z;
    if (s == 0.0f || R.nt == 0) return false;
    const float x = X / s, y = Y / s;
    if (!(x >= -0.3f && x <= 1.0f && y >= -0.3f && y <= 1.2f)) return false;
    int best = -1;
    float bw[3] = {0, 0, 0}, best_min = -INFINITY;
    for (int t = 0; t < R.nt; ++t) {
        const int i0 = R.tris[3 * t], i1 = R.tris[3 * t + 1], i2 = R.tris[3 * t + 2];
        const float ax = R.points[2 * i0], ay = R.points[2 * i0 + 1];
        const float bx = R.points[2 * i1], by = R.points[2 * i1 + 1];
        const float qx = R.points[2 * i2], qy = R.points[2 * i2 + 1];
        const float det = (bx - ax) * (qy - ay) - (qx - ax) * (by - ay);
        if (det == 0.0f) continue;
        const float w1 = ((x - ax) * (qy - ay) - (qx - ax) * (y - ay)) / det;
        const float w2 = ((bx - ax) * (y - ay) - (x - ax) * (by - ay)) / det;
        const float w0 = 1.0f - w1 - w2;
        const float mn = std::min(w0, std::min(w1, w2));
        if (mn > best_min) {
            best_min = mn;
            best = t;
            bw[0] = w0;
            bw[1] = w1;
            bw[2] = w2;
        }
    }
    if (best < 0) return false;
    float wtot = 0;
    for (int j = 0; j < 3; ++j) {
        const int i = R.tris[3 * best + j];
        idx[j] = i < R.ns ? i : -1;
        if (idx[j] < 0) bw[j] = 0;
        wtot += bw[j];
    }
    if (wtot == 0) return false;
    for (int j = 0; j < 3; ++j) w[j] = bw[j] * (s / wtot);
    return true;
}

// RecoveryMengSimon::doRecover (Single mode) at lam: the blend interpolated between the table's
// wavelengths; as a reflectance divided by the blend of the spectra's maxima when that exceeds 1
float rec_eval(const RecView& R, const int32_t idx[3], const float w[3], float lam, bool reflectant) {
    const float* ws = R.wavelengths;
    const int k = (int)(std::upper_bound(ws, ws + R.nw, lam) - ws);
    if (k == 0 || k == R.nw) return 0.0f;
    const float t = (lam - ws[k - 1]) / (ws[k] - ws[k - 1]);
    float v0 = 0, v1 = 0, mx = 0;
    for (int j = 0; j < 3; ++j) {
        if (idx[j] < 0) continue;
        const float* sp = R.spectra + (size_t)idx[j] * R.nw;
        v0 += w[j] * sp[k - 1];
        v1 += w[j] * sp[k];
        mx += w[j] * *std::max_element(sp, sp + R.nw);
    }
    const float v = v0 + t * (v1 - v0);
    return reflectant && mx > 1.0f ? v / mx : v;
}

// the point a texture is looked up at: (u, v), its screen-space derivatives, the squared surface
// footprint and the hit point
struct TexPoint {
    float u, v, du_i, dv_i, du_j, dv_j, fp2;
    V x;
};
TexPoint tp(const Ctx& c) { return TexPoint{c.uv_u, c.uv_v, c.du_i, c.dv_i, c.du_j, c.dv_j, c.fp2, c.target}; }

// Image::mipMapLevel (image.cpp:580-612): level maxLevel + log2(width), the fraction from the
// significand
void mip_level(float width, int n_levels, int& l0, int& l1, float& frac_) {
    const int max_level = n_levels - 1;
    const float w = std::max(width, 1e-9f);
    int32_t i;
    std::memcpy(&i, &w, 4);
    const int level = max_level + ((i >> 23) - 127);
    if (level < 0) {
        l0 = l1 = 0;
        frac_ = 0;
    } else if (level >= max_level) {
        l0 = l1 = max_level;
        frac_ = 0;
    } else {
        l0 = level;
        l1 = level + 1;
        const int32_t mi = (127 << 23) | (i & 0x7fffff);
        float m;
        std::memcpy(&m, &mi, 4);
        frac_ = m - 1.0f;
    }
}

// level (iu, iv) of an image's mip table at texture_pixels[T.pixels] (include/liar_gpu.h)
struct MipLevel {
    const float* px;
    int w, h;
};
MipLevel mip_get(const Scene& S, const Texture& T, int n_u, int iu, int iv) {
    const float* base = S.in.texture_pixels + 4 * T.pixels;
    int32_t e[4];
    std::memcpy(e, base + 4 * (1 + iv * n_u + iu), sizeof(e));
    const uint64_t off = ((uint64_t)(uint32_t)e[1] << 31) | (uint64_t)(uint32_t)e[0];
    return MipLevel{base + 4 * off, e[2], e[3]};
}

// Image::nearest (image.cpp:618-631) and Image::bilinear (image.cpp:636-690, the vectorised
// build): (u, 1 - v) with wrap-around
void image_nearest(const MipLevel& m, float u, float v, float out[3]) {
    int x0 = (int)std::floor(frac(u) * (float)m.w), y0 = (int)std::floor(frac(1.0f - v) * (float)m.h);
    x0 = std::min(std::max(x0, 0), m.w - 1);
    y0 = std::min(std::max(y0, 0), m.h - 1);
    for (int c = 0; c < 3; ++c) out[c] = m.px[4 * ((size_t)y0 * m.w + x0) + c];
}
void image_bilinear(const MipLevel& m, float u, float v, float out[3]) {
    const float x = frac(u) * (float)m.w - 0.5f, y = frac(1.0f - v) * (float)m.h - 0.5f;
    const float x0 = std::floor(x), y0 = std::floor(y), dx = x - x0, dy = y - y0;
    int i0 = (int)x0, j0 = (int)y0;
    if (i0 < 0) i0 += m.w;
    if (j0 < 0) j0 += m.h;
    i0 = std::min(std::max(i0, 0), m.w - 1);
    j0 = std::min(std::max(j0, 0), m.h - 1);
    const int i1 = i0 + 1 < m.w ? i0 + 1 : 0, j1 = j0 + 1 < m.h ? j0 + 1 : 0;
    for (int c = 0; c < 3; ++c) {
        const float p00 = m.px[4 * ((size_t)j0 * m.w + i0) + c], p10 = m.px[4 * ((size_t)j0 * m.w + i1) + c];
        const float p01 = m.px[4 * ((size_t)j1 * m.w + i0) + c], p11 = m.px[4 * ((size_t)j1 * m.w + i1) + c];
        const float a = (1 - dx) * p00 + dx * p10, b = (1 - dx) * p01 + dx * p11;
        out[c] = (1 - dy) * a + dy * b;
    }
}

// Image::lookUp (image.cpp:249-330): levels from the footprint, then nearest, bilinear, or
// trilinear across the levels
void image_lookup(const Scene& S, const Texture& T, const TexPoint& q, float out[3]) {
    int32_t hdr[4];
    std::memcpy(hdr, S.in.texture_pixels + 4 * T.pixels, sizeof(hdr));
    const int n_u = hdr[0], n_v = hdr[1], mip = hdr[2];
    int u0 = 0, u1 = 0, v0 = 0, v1 = 0;
    float fu = 0, fv = 0;
    const float wu = std::max(std::fabs(q.du_i), std::fabs(q.du_j)), wv = std::max(std::fabs(q.dv_i), std::fabs(q.dv_j));
    if (mip == 1) {
        mip_level(std::max(wu, wv), n_u, u0, u1, fu);
    } else if (mip == 2) {
        mip_level(wu, n_u, u0, u1, fu);
        mip_level(wv, n_v, v0, v1, fv);
    }
    const int aa = (int)T.p[0];
    if (aa == 0) return image_nearest(mip_get(S, T, n_u, u0, v0), q.u, q.v, out);
    if (aa == 1) return image_bilinear(mip_get(S, T, n_u, u0, v0), q.u, q.v, out);
    float p00[3], p10[3];
    image_bilinear(mip_get(S, T, n_u, u0, v0), q.u, q.v, p00);
    image_bilinear(mip_get(S, T, n_u, u1, v0), q.u, q.v, p10);
    for (int c = 0; c < 3; ++c) out[c] = (1 - fu) * p00[c] + fu * p10[c];
    if (v0 != v1) {
        float p01[3], p11[3];
        image_bilinear(mip_get(S, T, n_u, u0, v1), q.u, q.v, p01);
        image_bilinear(mip_get(S, T, n_u, u1, v1), q.u, q.v, p11);
        for (int c = 0; c < 3; ++c) out[c] = (1 - fv) * out[c] + fv * ((1 - fu) * p01[c] + fu * p11[c]);
    }
}

// CheckerBoard::weightA and ::integrate (checker_board.cpp:149-207): the share of A over the
// footprint's (u, v) box with bilinear anti-aliasing, else (or for an empty box) the point rule
float checker_weight(const Texture& T, const TexPoint& q) {
    const float sx = T.p[0], sy = T.p[1];
    const float fu = frac(q.u), fv = frac(q.v);
    const float point = (fu < sx) == (fv < sy) ? 1.0f : 0.0f;
    if (T.p[2] == 0.0f) return point;
    const float du = std::max(std::fabs(q.du_i), std::fabs(q.du_j)), dv = std::max(std::fabs(q.dv_i), std::fabs(q.dv_j));
    const float area = du * dv;
    if (!(area > 0.0f)) return point;
    const float mn[2] = {fu - du / 2, fv - dv / 2}, mx[2] = {fu + du / 2, fv + dv / 2};
    const float split[2] = {sx, sy};
    float d0[2], cmin[2][2], cmax[2][2];  // cmin[axis] = (min(d, split), max(d - split, 0)) of the low corner
    for (int k = 0; k < 2; ++k) {
        const float a0 = std::floor(mn[k]), b0 = std::floor(mx[k]);
        d0[k] = b0 - a0;
        const float dmn = mn[k] - a0, dmx = mx[k] - b0;
        cmin[k][0] = std::min(dmn, split[k]);
        cmin[k][1] = std::max(dmn - split[k], 0.0f);
        cmax[k][0] = std::min(dmx, split[k]);
        cmax[k][1] = std::max(dmx - split[k], 0.0f);
    }
    const float oneU[2] = {sx, 1 - sx}, oneV[2] = {sy, 1 - sy};
    auto dot2 = [](const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1]; };
    float r = (sx * sy + (1 - sx) * (1 - sy)) * d0[0] * d0[1];
    r += (dot2(oneU, cmax[1]) - dot2(oneU, cmin[1])) * d0[0];
    r += (dot2(cmax[0], oneV) - dot2(cmin[0], oneV)) * d0[1];
    r += dot2(cmax[0], cmax[1]) - dot2(cmax[0], cmin[1]);
    r += dot2(cmin[0], cmin[1]) - dot2(cmin[0], cmax[1]);
    return std::min(std::max(r / area, 0.0f), 1.0f);
}

// Texture::lookUp of the uv textures (src/liar/textures/): TransformationUv moves the context's uv
// (transformation_uv.cpp:67-70), CheckerBoard without anti-aliasing picks A where the fractional u
// and v lie on the same side of the split (checker_board.cpp:113-124, 149-157), GridBoard picks A
// on the lines (grid_board.cpp:80-87), Constant is its spectrum
// Perlin::noise and FBm::doScalarLookUp (perlin.cpp:60-90, 170-205; fbm.cpp:62-90 with a zero
// footprint, so every octave): improved Perlin noise on a 256-periodic lattice
float perlin_gradient(const uint8_t* tab, int x, int y, int z, float dx, float dy, float dz) {
    static const int8_t G[16][3] = {{1, 1, 0}, {-1, 1, 0}, {1, -1, 0}, {-1, -1, 0}, {1, 0, 1}, {-1, 0, 1},
                                    {1, 0, -1}, {-1, 0, -1}, {0, 1, 1}, {0, -1, 1}, {0, 1, -1}, {0, -1, -1},
                                    {1, 1, 0}, {-1, 1, 0}, {0, -1, 1}, {0, -1, -1}};
    const int8_t* g = G[(tab[x] ^ tab[257 + y] ^ tab[514 + z]) & 15];
    float r = 0;  // the reference's sums, term by term in its order
    const float c[3] = {dx, dy, dz};
    int first = -1;
    for (int k = 0; k < 3; ++k)
        if (g[k] != 0 && first < 0) first = k;
    r = g[first] * c[first];
    for (int k = first + 1; k < 3; ++k)
        if (g[k] != 0) r = r + g[k] * c[k];
    return r;
}

float perlin_noise(const uint8_t* tab, V q) {
    const float c[3] = {q.x, q.y, q.z};
    float d[3];
    int i[3];
    for (int k = 0; k < 3; ++k) {
        const float m = c[k] - std::floor(c[k] * (1.0f / 256.0f)) * 256.0f;
        const float f = std::floor(m);
        i[k] = (int)f;
        d[k] = m - f;
        if (i[k] >= 256 || i[k] < 0) i[k] = 0;
    }
    float g[8];
    for (int n = 0; n < 8; ++n) {
        const int a = n & 1, b = (n >> 1) & 1, e = (n >> 2) & 1;
        g[n] = perlin_gradient(tab, i[0] + a, i[1] + b, i[2] + e, d[0] - a, d[1] - b, d[2] - e);
    }
    auto fade = [](float x) { const float x2 = x * x; return (6 * x2 * x - 15 * x2 + 10 * x) * x2; };
    auto lerp = [](float a, float b, float t) { return a + t * (b - a); };
    const float sx = fade(d[0]), sy = fade(d[1]), sz = fade(d[2]);
    return lerp(lerp(lerp(g[0], g[1], sx), lerp(g[2], g[3], sx), sy), lerp(lerp(g[4], g[5], sx), lerp(g[6], g[7], sx), sy),
                sz);
}

// FBm::doScalarLookUp (fbm.cpp:76-101): 1 - log2(footprint^2) / 2 octaves clamped to [1, octaves],
// the last one's fraction blended in; Perlin when p[0] = 0
float noise_texture(const Scene& S, const Texture& T, const TexPoint& q) {
    const uint8_t* tab = S.in.noise_tables + T.pixels;
    const int octaves = (int)T.p[0];
    if (octaves <= 0) return perlin_noise(tab, q.x);
    const float ideal = 1.0f - std::log2(q.fp2) / 2.0f;
    const float real = std::min(std::max(ideal, 1.0f), (float)octaves);
    const int n = (int)std::floor(real);
    float result = 0, freq = 1, weight = 1;
    for (int k = 0; k < n; ++k) {
        result += weight * perlin_noise(tab, freq * q.x);
        freq *= 2;
        weight *= T.p[1];
    }
    const float fr = real - (float)n;
    if (fr > 0) result += fr * weight * perlin_noise(tab, freq * q.x);
    return result;
}

// Abs (abs.cpp:26-35) looks its input up as the caller does; Product / Sum of one texture with
// constants (product.cpp:90-99, sum.cpp:90-105) as illuminants, the result clamped as a
// reflectance; applied to the value found below them
float texture_rec(const Scene& S, int t, TexPoint q, float lam, bool reflectant, int depth0) {
    for (int depth = depth0; depth < 64; ++depth) {
        const Texture& T = S.in.textures[t];
        if (T.type == 1) {
            const float wa = checker_weight(T, q);
            if (wa >= 1) {
                t = T.a;
            } else if (wa <= 0) {
                t = T.b;
            } else {
                // Spectral(wA A + (1 - wA) B, type) of the two looked up as illuminants
                const float va = texture_rec(S, T.a, q, lam, false, depth + 1);
                const float vb = texture_rec(S, T.b, q, lam, false, depth + 1);
                const float r = wa * va + (1 - wa) * vb;
                return reflectant ? std::min(r, 1.0f) : r;
            }
        } else if (T.type == 2) {
            const float fu = frac(q.u), fv = frac(q.v);
            t = (fu < T.p[0] || fv < T.p[0] || fu > 1 - T.p[0] || fv > 1 - T.p[1]) ? T.a : T.b;
        } else if (T.type == 3) {
            // TransformationUv (transformation_uv.cpp:67-70): (u, v) and its derivatives
            TexPoint n = q;
            n.u = T.p[0] * q.u + T.p[1] * q.v + T.p[2];
            n.v = T.p[3] * q.u + T.p[4] * q.v + T.p[5];
            n.du_i = T.p[0] * q.du_i + T.p[1] * q.dv_i;
            n.dv_i = T.p[3] * q.du_i + T.p[4] * q.dv_i;
            n.du_j = T.p[0] * q.du_j + T.p[1] * q.dv_j;
            n.dv_j = T.p[3] * q.du_j + T.p[4] * q.dv_j;
            q = n;
            t = T.a;
        } else if (T.type == 5) {
            const float n = noise_texture(S, T, q);
            return reflectant ? std::min(n, 1.0f) : n;
        } else if (T.type == 6) {
            return std::fabs(texture_rec(S, T.a, q, lam, reflectant, depth + 1));
        } else if (T.type == 7) {
            const float r = T.p[0] * texture_rec(S, T.a, q, lam, false, depth + 1) + T.p[1];
            return reflectant ? std::min(r, 1.0f) : r;
        } else if (T.type == 4) {
            // Image::doLookUp: Spectral::fromXYZ of the colour
            float c[3];
            image_lookup(S, T, q, c);
            int32_t idx[3];
            float w[3];
            if (!rec_locate(S.rec, c[0], c[1], c[2], idx, w)) return 0;
            return rec_eval(S.rec, idx, w, lam, reflectant);
        } else {
            return spectrum(S, T.spectrum, lam, reflectant);
        }
    }
    return 0;
}

float param(const Scene& S, const Material& M, int k, const TexPoint& q, float lam, bool reflectant) {
    return M.tex[k] >= 0 ? texture_rec(S, M.tex[k], q, lam, reflectant, 0) : spectrum(S, M.spec[k], lam, reflectant);
}
Ctx hit_ctx(const Scene& S, V o, V d, const Hit& h) {
    Ctx c;
    const uint32_t prim = (uint32_t)h.prim;
    if (prim >= S.in.n_triangles) {
        // Sphere::doLocalContext (sphere.cpp:130-175): the point reprojected onto the surface, the
        // outward normal, uv of its spherical angles, dPoint/du along (-n.y, n.x, 0)
        const uint64_t k = prim - S.in.n_triangles;
        const float* sp = S.in.spheres + 4 * k;
        const V C{sp[0], sp[1], sp[2]};
        c.obj = S.in.sphere_object[k];
        c.light = S.in.object_light[c.obj];
        c.mi = S.in.object_material[c.obj];
        const V n0 = unit((o + h.t * d) - C);
        c.target = C + sp[3] * n0;
        c.uv_u = std::atan2(n0.y, n0.x) * (0.5f / 3.14159265358979323846f);
        c.uv_v = std::acos(std::min(std::max(n0.z, -1.0f), 1.0f)) * (1.0f / 3.14159265358979323846f);
        c.leaving = dot(d, n0) > 0;
        c.ng = dot(n0, -d) < 0 ? -n0 : n0;
        c.N = c.ng;
        V u{-n0.y, n0.x, 0.0f};
        u = u - dot(u, c.N) * c.N;
        if (dot(u, u) < 1e-12f) u = cross(std::fabs(c.N.x) < 0.9f ? V{1, 0, 0} : V{0, 1, 0}, c.N);
        c.u = unit(u);
        c.v = cross(c.N, c.u);
        return c;
    }
    c.obj = S.in.triangle_object[prim];
    c.light = S.in.object_light[c.obj];
    c.mi = S.in.object_material[c.obj];
    const uint32_t* tr = S.in.triangles + 3 * (size_t)prim;
    const float* pa = S.in.vertices + 3 * tr[0];
    const float* pb = S.in.vertices + 3 * tr[1];
    const float* pc = S.in.vertices + 3 * tr[2];
    const V A{pa[0], pa[1], pa[2]};
    const V e1 = V{pb[0], pb[1], pb[2]} - A, e2 = V{pc[0], pc[1], pc[2]} - A;
    float tt, bu = 0, bv = 0;
    const float oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
    if (!oracle_tri_intersect(oo, dd, pa, pb, pc, &tt, &bu, &bv)) bu = bv = 0;
    c.target = A + bu * e1 + bv * e2;
    hit_uv(S, prim, bu, bv, c.uv_u, c.uv_v);
    const V ng0 = unit(cross(e1, e2));
    V ns = ng0;
    if (S.in.triangle_normals && S.in.normals) {
        const int32_t* tn = S.in.triangle_normals + 3 * (size_t)prim;
        if (tn[0] >= 0 && tn[1] >= 0 && tn[2] >= 0) {
            const float* n0 = S.in.normals + 3 * tn[0];
            const float* n1 = S.in.normals + 3 * tn[1];
            const float* n2 = S.in.normals + 3 * tn[2];
            const float w0 = 1 - bu - bv;
            ns = unit(w0 * V{n0[0], n0[1], n0[2]} + bu * V{n1[0], n1[1], n1[2]} + bv * V{n2[0], n2[1], n2[2]});
        }
    }
    c.leaving = dot(d, ng0) > 0;
    c.ng = dot(ng0, -d) < 0 ? -ng0 : ng0;  // flipTo(-direction)
    c.N = dot(ns, -d) < 0 ? -ns : ns;
    // frame: IntersectionContext::bsdfToLocal
    V u = e1 - dot(e1, c.N) * c.N, v = e2 - dot(e2, c.N) * c.N;
    const float su = dot(u, u), sv = dot(v, v);
    if (std::max(su, sv) < 1e-3f * std::max(dot(e1, e1), dot(e2, e2))) {
        const V ax = std::fabs(c.N.x) < 0.9f ? V{1, 0, 0} : V{0, 1, 0};
        u = cross(ax, c.N);
        v = cross(c.N, u);
    }
    if (su >= sv) {
        u = unit(u);
        v = cross(c.N, u);
    } else {
        v = unit(v);
        u = cross(v, c.N);
    }
    c.u = u;
    c.v = v;
    return c;
}

// Shader::bsdf at one wavelength
Bsdf make_bsdf(const Scene& S, const Material& M, const Ctx& c, float lam) {
    Bsdf B{};
    B.type = M.type;
    B.mdf = M.mdf;
    B.ng = {dot(c.ng, c.u), dot(c.ng, c.v), dot(c.ng, c.N)};
    B.eta = B.kappa = B.ior = B.etaI = B.etaT = 1;
    B.au = sq(std::max(M.rough_u, 1e-3f));
    B.av = sq(std::max(M.rough_v, 1e-3f));
    switch (M.type) {
        case M_LAMBERT:
            B.caps = C_REFL | C_DIFF;
            B.r = param(S, M, 0, tp(c), lam, true);
            break;
        case M_CONDUCTOR:
        case M_CT:
            B.caps = M.type == M_CONDUCTOR ? (C_REFL | C_SPEC) : (C_REFL | C_GLOSSY);
            B.eta = std::max(param(S, M, 0, tp(c), lam, false), 1e-9f);
            B.kappa = std::max(param(S, M, 1, tp(c), lam, false), 1e-9f);
            B.r = param(S, M, 2, tp(c), lam, true);
            break;
        case M_DIELECTRIC: {
            B.caps = C_REFL | C_TRANS | C_SPEC;
            const float i1 = std::max(param(S, M, 1, tp(c), lam, false), 1e-9f);
            const float i2 = std::max(param(S, M, 0, tp(c), lam, false), 1e-9f);
            B.ior = c.leaving ? i2 / i1 : i1 / i2;
            B.r = param(S, M, 2, tp(c), lam, true);
            B.t = param(S, M, 3, tp(c), lam, true);
            break;
        }
        case M_WALTER: {
            B.caps = C_TRANS | C_GLOSSY;
            float ei = std::max(param(S, M, 1, tp(c), lam, false), 1e-9f);
            float et = std::max(param(S, M, 0, tp(c), lam, false), 1e-9f);
            if (c.leaving) std::swap(ei, et);
            B.etaI = ei;
            B.etaT = et;
            B.r = param(S, M, 2, tp(c), lam, true);
            B.t = param(S, M, 3, tp(c), lam, true);
            break;
        }
        case M_MIRROR:
            B.caps = C_REFL | C_SPEC;
            B.r = param(S, M, 0, tp(c), lam, true);
            break;
    }
    return B;
}

// PerspectiveCamera::doGenerateRay (perspective_camera.cpp:406-434) at screen point (sx, sy) and
// lens sample (lu, lv)
void camera_at(const Camera& C, float sx, float sy, float lu, float lv, V& pos, V& dir, float& factor) {
    pos = V{C.position[0], C.position[1], C.position[2]};
    dir = V{C.direction[0], C.direction[1], C.direction[2]} + (sx - 0.5f) * V{C.right[0], C.right[1], C.right[2]} +
          (sy - 0.5f) * V{C.down[0], C.down[1], C.down[2]};
    dir = unit(dir);
    const V dn{C.direction_normal[0], C.direction_normal[1], C.direction_normal[2]};
    factor = 1 / dot(dir, dn);
    if (C.lens_radius > 0 && C.focus_distance > 0 && C.focus_distance < 3.4e38f) {
        float lx, ly;
        concentric(lu, lv, lx, ly);
        const V lp = pos + (C.lens_radius * lx) * V{C.right_normal[0], C.right_normal[1], C.right_normal[2]} +
                     (C.lens_radius * ly) * V{C.down_normal[0], C.down_normal[1], C.down_normal[2]};
        const V fp = pos + (factor * C.focus_distance) * dir;
        pos = lp;
        dir = unit(fp - lp);
        factor = 1 / dot(dir, dn);
    }
}

void camera_samples(const RenderIn& R, const Sampler& smp, float& sx, float& sy, float& lu, float& lv) {
    const uint32_t ix = smp.pixel % (uint32_t)R.width, iy = smp.pixel / (uint32_t)R.width;
    float jx, jy;
    smp.get2(D_SCREEN, jx, jy);
    sx = ((float)ix + jx) / (float)R.width;
    sy = ((float)iy + jy) / (float)R.height;
    smp.get2(D_LENS, lu, lv);
}

// dPoint/du and dPoint/dv of the hit's parametrisation (corner uvs, else the barycentrics; a
// sphere's spherical angles, sphere.cpp:150-172)
bool hit_dpduv(const Scene& S, uint32_t prim, V n_out, V& dpdu, V& dpdv) {
    if (prim >= S.in.n_triangles) {
        const float r = S.in.spheres[4 * (prim - S.in.n_triangles) + 3];
        const float pi = 3.14159265358979323846f;
        const float theta = std::acos(std::min(std::max(n_out.z, -1.0f), 1.0f));
        const float st = std::sin(theta);
        dpdu = (r * 2.0f * pi) * V{-n_out.y, n_out.x, 0.0f};
        if (st != 0.0f) {
            const float cs = n_out.z / st;
            dpdv = (r * pi) * V{cs * n_out.x, cs * n_out.y, -st};
        } else {
            const float phi = std::atan2(n_out.y, n_out.x);
            dpdv = (r * pi) * V{std::cos(phi), std::sin(phi), 0.0f};
        }
        return true;
    }
    const uint32_t* tr = S.in.triangles + 3 * (size_t)prim;
    const float* pa = S.in.vertices + 3 * tr[0];
    const float* pb = S.in.vertices + 3 * tr[1];
    const float* pc = S.in.vertices + 3 * tr[2];
    const V A{pa[0], pa[1], pa[2]};
    const V e1 = V{pb[0], pb[1], pb[2]} - A, e2 = V{pc[0], pc[1], pc[2]} - A;
    if (!S.in.triangle_uvs) {
        dpdu = e1;
        dpdv = e2;
        return true;
    }
    const float* t = S.in.triangle_uvs + 6 * (size_t)prim;
    const float du1 = t[2] - t[0], dv1 = t[3] - t[1], du2 = t[4] - t[0], dv2 = t[5] - t[1];
    const float det = du1 * dv2 - dv1 * du2;
    if (det == 0.0f) return false;
    const float inv = 1.0f / det;
    dpdu = inv * (dv2 * e1 - dv1 * e2);
    dpdv = inv * (du1 * e2 - du2 * e1);
    return true;
}

// IntersectionContext::setScreenSpaceDifferentialsI (intersection_context.cpp:295-324) for the
// camera's two differential rays (Camera::primaryRay, camera.cpp:53-60: the screen point moved by
// 1 / (resolution sqrt(spp)), render_engine.cpp:211-215): where each meets the tangent plane, and
// the (u, v) step of that offset on the plane's two minor axes (Cramer's rule)
void camera_footprint(const Scene& S, const RenderIn& R, const Sampler& smp, uint32_t prim, Ctx& c) {
    float sx, sy, lu, lv, f;
    camera_samples(R, smp, sx, sy, lu, lv);
    const float root = std::sqrt((float)smp.spp);
    const float dsx = 1.0f / ((float)R.width * root), dsy = 1.0f / ((float)R.height * root);
    V oi, di, oj, dj;
    camera_at(R.camera, sx + dsx, sy, lu, lv, oi, di, f);
    camera_at(R.camera, sx, sy + dsy, lu, lv, oj, dj, f);
    V n_out = c.N;
    if (prim >= S.in.n_triangles) {
        const float* sp = S.in.spheres + 4 * (prim - S.in.n_triangles);
        n_out = unit(c.target - V{sp[0], sp[1], sp[2]});
    }
    V dpdu, dpdv;
    if (!hit_dpduv(S, prim, n_out, dpdu, dpdv)) return;
    const V N = c.N, P = c.target;
    const float ax = std::fabs(N.x), ay = std::fabs(N.y), az = std::fabs(N.z);
    const int major = ax >= ay ? (ax >= az ? 0 : 2) : (ay >= az ? 1 : 2);
    const int a = (major + 1) % 3, b = (major + 2) % 3;
    auto comp = [](V v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); };
    const float m00 = comp(dpdu, a), m01 = comp(dpdv, a), m10 = comp(dpdu, b), m11 = comp(dpdv, b);
    const float det = m00 * m11 - m01 * m10;
    float fp2 = 0;
    for (int side = 0; side < 2; ++side) {
        const V o = side ? oj : oi, d = side ? dj : di;
        const float nd = dot(N, d);
        if (nd == 0.0f) continue;
        const float t = dot(N, P - o) / nd;
        if (!(t >= 0.0f)) continue;
        const V dp = (o + t * d) - P;
        fp2 = std::max(fp2, dot(dp, dp));
        if (det == 0.0f) continue;
        const float ra = comp(dp, a), rb = comp(dp, b);
        const float du = (ra * m11 - m01 * rb) / det, dv = (m00 * rb - ra * m10) / det;
        (side ? c.du_j : c.du_i) = du;
        (side ? c.dv_j : c.dv_i) = dv;
    }
    c.fp2 = fp2;
}

// AdjointPhotonTracer::shadeSurface + scatterSurface for the hit `h` of ray (o, d)
float shade_surface(Path& P, V o, V d, float tmin, float tmax, const Hit& h, int gen) {
    const Scene& S = *P.S;
    float result = 0;
    Ctx c = hit_ctx(S, o, d, h);
    if (gen == 0 && S.in.n_textures > 0) camera_footprint(S, *P.R, P.smp, (uint32_t)h.prim, c);  // the camera vertex
    const int light = c.light, mi = c.mi;
    const V target = c.target, ng = c.ng, N = c.N, u = c.u, v = c.v;
    if (gen > 0 && light >= 0) result += spectrum(S, S.in.lights[light].spectrum, P.lam, false);
    // the shader's emission counts unless the object is a light hit past the camera vertex
    // (shadeSurface asks for the object's light only at generations > 0)
    const bool shader_emits = gen == 0 || light < 0;
    if (mi < 0) return result + trace_photon(P, o, d, h.t + TOL, tmax, gen + 1);  // no shader: continue through
    if (S.in.materials[mi].type == M_NONE) {
        // a shader without a BSDF: its emission, nothing scatters
        if (shader_emits && S.in.materials[mi].emission >= 0) result += spectrum(S, S.in.materials[mi].emission, P.lam, false);
        return result;
    }
    const Material& M = S.in.materials[mi];
    if (shader_emits && M.emission >= 0) result += spectrum(S, M.emission, P.lam, false);
    const Bsdf B = make_bsdf(S, M, c, P.lam);
    const V md = -d;
    V wi{dot(md, u), dot(md, v), dot(md, N)};
    wi.z = std::max(wi.z, 1.19209290e-07f);
    // scatterSurface
    const bool strat = gen < P.R->max_ray_generation;
    const uint32_t base = D_GEN0 + D_PER_GEN * (uint32_t)gen;
    const float spdf = (has(B.caps, C_DIFF) || has(B.caps, C_GLOSSY)) ? 0.5f : 1.0f;
    Out out{{0, 0, 0}, 0, 0};
    if (P.smp.get(base + O_STRAT, strat) < spdf) {
        out = sample(B, wi, P.smp.get(base + O_BSDF, strat), P.smp.get(base + O_BSDF + 1, strat),
                     P.smp.get(base + O_COMP, strat), C_ALL);
        if (!out) return result;
        out.pdf *= spdf;
        const V wd = out.wo.x * u + out.wo.y * v + out.wo.z * N;
        float pl = 0;
        for (int l = 0; l < (int)S.in.n_lights; ++l) {
            const float p = light_emission_pdf(S, l, target, wd);
            if (p > 0) pl += light_pdf_choice(S, l) * p;
        }
        pl *= (1 - spdf);
        out.value *= power_heuristic(out.pdf, pl);
    } else {
        if (S.in.n_lights == 0) return result;
        const float uc = P.smp.get(base + O_LCHOICE, strat);
        int k = (int)(std::lower_bound(S.light_cdf.begin(), S.light_cdf.end(), uc) - S.light_cdf.begin());
        k = std::min(k, (int)S.in.n_lights - 1);
        const float pc = light_pdf_choice(S, k);
        if (pc <= 0) return result;
        const LS ls = light_sample(S, k, target, P.smp.get(base + O_LIGHT, strat), P.smp.get(base + O_LIGHT + 1, strat));
        if (ls.pdf <= 0) return result;
        float pdf = pc * ls.pdf;
        for (int l = 0; l < (int)S.in.n_lights; ++l) {
            if (l == k) continue;
            const float p = light_emission_pdf(S, l, target, ls.dir);
            if (p > 0) pdf += light_pdf_choice(S, l) * p;
        }
        pdf *= (1 - spdf);
        const V wo{dot(ls.dir, u), dot(ls.dir, v), dot(ls.dir, N)};
        const Out be = evaluate(B, wi, wo, C_ALL);
        if (!be) return result;
        out = {wo, be.value * power_heuristic(pdf, be.pdf * spdf), pdf};
    }
    if (!out) return result;
    const float ct = out.wo.z;
    const V start = target + ((ct > 0 ? 10.0f : -10.0f) * TOL) * ng;
    const V nd = out.wo.x * u + out.wo.y * v + out.wo.z * N;
    const float radiance = trace_photon(P, start, nd, TOL, INFINITY, gen + 1);
    return result + (out.value * radiance) * (std::fabs(ct) / out.pdf);
}

float trace_photon(Path& P, V o, V d, float tmin, float tmax, int gen) {
    const Scene& S = *P.S;
    float power = 1;
    if (P.R->max_depth > 0 && gen >= P.R->max_depth) return 0;
    if (gen >= P.R->max_ray_generation) {
        const float u = P.smp.get(D_GEN0 + D_PER_GEN * (uint32_t)gen + O_RR, false);
        if (u < 0.5f) power /= 0.5f;
        else return 0;
    }
    const Hit h = oracle_internal::tree_closest(S.tree, Ray{o.x, o.y, o.z, tmin, d.x, d.y, d.z, tmax});
    if (h.prim < 0) {
        if (S.sky >= 0 && S.sky_distance > tmin * (1 + TOL) && S.sky_distance < tmax * (1 - TOL)) {
            if (gen == 0) P.alpha = 1;
            if (gen > 0) return power * spectrum(S, S.in.lights[S.sky].spectrum, P.lam, false);
        }
        return 0;
    }
    if (gen == 0) P.alpha = 1;
    return power * shade_surface(P, o, d, tmin, tmax, h, gen);
}

// ---- DirectLighting (tracers/direct_lighting.cpp) with RayTracer::estimateLightContribution
// (kernel/ray_tracer.cpp:188-276): the recursive form of the library's wavefront (csrc/direct.cu),
// with the same sample dimensions, branch keys and shadow-ray bounds.
const float SHADOW_SHRINK = 1e-4f;

uint32_t dl_dim_light(int l, int k, int axis) { return 0x200000u + ((uint32_t)l * 1024u + (uint32_t)k) * 8u + (uint32_t)axis; }
uint32_t dl_dim_scatter(int i, int axis) { return 0x400000u + (uint32_t)i * 8u + (uint32_t)axis; }
uint32_t dl_dim_branch(uint32_t key, uint32_t j) {
    return 0x80000000u | (uint32_t)(mix64(((uint64_t)key << 20) ^ j) & 0x7fffffffu);
}
uint32_t dl_child_key(uint32_t key, uint32_t c) { return (uint32_t)mix64(((uint64_t)key << 8) | (c + 1u)) | 1u; }

// SceneLight::sampleEmission: direction, distance, solid-angle pdf, radiance
struct LSF {
    V dir;
    float dist, pdf, value;
};
LSF light_sample_full(const Scene& S, int li, V target, float sx, float sy, float lam) {
    const Light& L = S.in.lights[li];
    const LS ls = light_sample(S, li, target, sx, sy);
    LSF out{ls.dir, 0, ls.pdf, 0};
    if (L.type == L_PARA || L.type == L_MESH) {
        // the sampled point again, for the distance (light_sample normalised the direction)
        V p;
        if (L.type == L_PARA) {
            p = V{L.pos[0], L.pos[1], L.pos[2]} + sx * V{L.u[0], L.u[1], L.u[2]} + sy * V{L.v[0], L.v[1], L.v[2]};
        } else {
            const float* cdf = S.tri_cdf.data() + L.first_tri;
            int ii = (int)(std::lower_bound(cdf, cdf + L.n_tris, sx) - cdf);
            ii = std::min(ii, L.n_tris - 1);
            const float i0 = ii > 0 ? cdf[ii - 1] : 0.0f;
            const float di = (sx - i0) / (cdf[ii] - i0);
            const uint32_t* tr = S.in.triangles + 3 * (size_t)(L.first_tri + ii);
            const float* a = S.in.vertices + 3 * tr[0];
            const float* b = S.in.vertices + 3 * tr[1];
            const float* c = S.in.vertices + 3 * tr[2];
            const float sr = std::sqrt(di);
            p = V{a[0], a[1], a[2]} + (1 - sr) * V{b[0] - a[0], b[1] - a[1], b[2] - a[2]} +
                (sr * sy) * V{c[0] - a[0], c[1] - a[1], c[2] - a[2]};
        }
        out.dist = len(p - target);
        if (out.pdf > 0) out.value = spectrum(S, L.spectrum, lam, false);
    } else if (L.type == L_POINT) {
        const V tl = V{L.pos[0], L.pos[1], L.pos[2]} - target;
        const float d2 = dot(tl, tl);
        out.dist = std::sqrt(d2);
        out.value = spectrum(S, L.spectrum, lam, false) / d2;
    } else if (L.type == L_SKY) {
        out.dist = S.sky_distance;
        out.value = spectrum(S, L.spectrum, lam, false);
    }
    return out;
}

// SceneLight::emission(ray): pdf, radiance and distance of the light along a direction
struct LEF {
    float pdf, value, t;
};
LEF light_emission_full(const Scene& S, int li, V o, V d, float lam) {
    const Light& L = S.in.lights[li];
    LEF e{0, 0, INFINITY};
    if (L.type == L_PARA) {
        float t;
        if (!para_hit(L, o, d, TOL, t)) return e;
        e.t = t;
    } else if (L.type == L_MESH) {
        float tb = INFINITY;
        for (int k = 0; k < L.n_tris; ++k) {
            const uint32_t* tr = S.in.triangles + 3 * (size_t)(L.first_tri + k);
            const float oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
            float t, uu, vv;
            if (oracle_tri_intersect(oo, dd, S.in.vertices + 3 * tr[0], S.in.vertices + 3 * tr[1],
                                     S.in.vertices + 3 * tr[2], &t, &uu, &vv) && t > TOL && t < tb)
                tb = t;
        }
        if (!(tb < INFINITY)) return e;
        e.t = tb;
    } else if (L.type == L_SKY) {
        e.t = S.sky_distance;
    } else {
        return e;
    }
    e.pdf = light_emission_pdf(S, li, o, d);
    if (e.pdf > 0) e.value = spectrum(S, L.spectrum, lam, false);
    return e;
}

struct DLPath {
    const Scene* S;
    const RenderIn* R;
    Sampler smp;
    float lam;
    float alpha = 0;
    const PmIn* pm = nullptr;  // PhotonMapper maps, nullptr for DirectLighting
};

// ---- PhotonMapper estimates (photon_mapper.cpp:1254-1381)

RecView pm_rec(const PmIn& pm) {
    RecView R;
    R.wavelengths = pm.rec_wavelengths;
    R.spectra = pm.rec_spectra;
    R.points = pm.rec_points;
    R.tris = pm.rec_tris;
    R.nw = pm.rec_nw;
    R.ns = pm.rec_ns;
    R.nt = pm.rec_nt;
    return R;
}
bool pm_locate(const PmIn& pm, float X, float Y, float Z, int32_t idx[3], float w[3]) {
    return rec_locate(pm_rec(pm), X, Y, Z, idx, w);
}
// Spectral::fromXYZ as an illuminant
float pm_recover(const PmIn& pm, const int32_t idx[3], const float w[3], float lam) {
    return rec_eval(pm_rec(pm), idx, w, lam, false);
}

// KdTree::rangeSearch(point, rMax, kMax): the k nearest photons with d^2 < rMax^2, by brute force
// (ascending d^2, ties by photon index)
void pm_nearest(const PmIn& pm, int m, V x, std::vector<std::pair<float, int64_t>>& out) {
    out.clear();
    const float r2max = pm.radius[m] * pm.radius[m];
    const float* P = pm.position[m];
    for (uint64_t i = 0; i < pm.n[m]; ++i) {
        const float dx = P[3 * i] - x.x, dy = P[3 * i + 1] - x.y, dz = P[3 * i + 2] - x.z;
        const float d2 = dx * dx + dy * dy + dz * dz;
        if (d2 < r2max) out.push_back({d2, (int64_t)i});
    }
    std::sort(out.begin(), out.end());
    if ((int64_t)out.size() > pm.k[m]) out.resize((size_t)pm.k[m]);
}

bool occluded(const Scene& S, V o, V d, float tmax) {
    return oracle_internal::tree_any(S.tree, Ray{o.x, o.y, o.z, TOL, d.x, d.y, d.z, tmax});
}

bool is_specular(const Bsdf& B) { return B.type == M_MIRROR || B.type == M_CONDUCTOR || B.type == M_DIELECTRIC; }

template <class U>
float estimate_light(const Scene& S, const Bsdf& B, const Ctx& c, V wi, V start, int l, int nl, int nb, float lam,
                     const U& u) {
    const Light& L = S.in.lights[l];
    const bool singular = L.type == L_POINT;
    uint32_t caps = C_REFL | C_TRANS | C_DIFF | C_GLOSSY;
    if (!singular) caps |= C_SPEC;
    const float fnl = (float)nl, fnb = (float)nb;
    float result = 0;
    for (int k = 0; k < nl; ++k) {
        const LSF ls = light_sample_full(S, l, start, u(0, k, 0), u(0, k, 1), lam);
        if (ls.pdf <= 0 || ls.value == 0) continue;
        if ((L.type == L_PARA || L.type == L_MESH) && dot(c.N, ls.dir) <= 0) continue;
        const V wo{dot(ls.dir, c.u), dot(ls.dir, c.v), dot(ls.dir, c.N)};
        const Out be = evaluate(B, wi, wo, caps);
        if (be.value == 0 || !(be.pdf > 0)) continue;
        if (occluded(S, start, ls.dir, ls.dist * (1 - SHADOW_SHRINK))) continue;
        const float w = power_heuristic(fnl * ls.pdf, fnb * be.pdf);
        result += be.value * ls.value * (w * std::fabs(wo.z) / (fnl * ls.pdf));
    }
    for (int k = 0; k < nb; ++k) {
        const Out bs = sample(B, wi, u(1, k, 0), u(1, k, 1), u(2, k, 0), caps);
        if (!bs) continue;
        const V wd = bs.wo.x * c.u + bs.wo.y * c.v + bs.wo.z * c.N;
        const LEF e = light_emission_full(S, l, start, wd, lam);
        if (!(e.pdf > 0) || e.value == 0) continue;
        if (occluded(S, start, wd, e.t * (1 - SHADOW_SHRINK))) continue;
        const float w = is_specular(B) ? 1.0f : power_heuristic(fnb * bs.pdf, fnl * e.pdf);
        result += bs.value * e.value * (w * std::fabs(bs.wo.z) / (fnb * bs.pdf));
    }
    return result;
}

// estimateRadiance (m = 0, global map, f without specular and glossy parts) and estimateCaustics
// (m = 1, caustic map, Gaussian filter, f's diffuse part): at least two photons, over pi r^2 with
// r^2 the farthest photon's squared distance
float pm_estimate(const DLPath& P, int m, const Ctx& c, const Bsdf& B, V wi) {
    const PmIn& pm = *P.pm;
    if (pm.n[m] == 0 || pm.k[m] < 1) return 0;
    thread_local std::vector<std::pair<float, int64_t>> nb;
    pm_nearest(pm, m, c.target, nb);
    if (nb.size() < 2) return 0;
    const float r2 = nb.back().first;
    if (!(r2 > 0)) return 0;
    const uint32_t caps = m == 0 ? (uint32_t)(C_ALL & ~C_SPEC & ~C_GLOSSY) : (uint32_t)(C_REFL | C_TRANS | C_DIFF);
    const float alpha = 0.918f, beta = 1.953f;
    const float b1 = -beta / (2.0f * r2), b2 = 1.0f / (1.0f - std::exp(-beta));
    float result = 0;
    for (const auto& e : nb) {
        const int64_t i = e.second;
        const float* om = pm.omega_in[m] + 3 * i;
        const V wo{om[0] * c.u.x + om[1] * c.u.y + om[2] * c.u.z, om[0] * c.v.x + om[1] * c.v.y + om[2] * c.v.z,
                   om[0] * c.N.x + om[1] * c.N.y + om[2] * c.N.z};
        const Out be = evaluate(B, wi, wo, caps);
        if (!(be.pdf > 0) || be.value == 0) continue;
        float v = be.value * pm_recover(pm, pm.blend_idx[m] + 3 * i, pm.blend_w[m] + 3 * i, P.lam);
        if (m == 1) v *= alpha * (1.0f - b2 * (1.0f - std::exp(b1 * e.first)));
        result += v;
    }
    return result / (3.14159265358979323846f * r2);
}

// isVisualizingPhotonMap: the global map's irradiance at the hit from the normal's side
// (estimateIrradianceImpl, photon_mapper.cpp:1254-1279) as a spectrum at lam
float pm_irradiance(const DLPath& P, const Ctx& c) {
    const PmIn& pm = *P.pm;
    if (pm.n[0] == 0 || pm.k[0] < 1) return 0;
    thread_local std::vector<std::pair<float, int64_t>> nb;
    pm_nearest(pm, 0, c.target, nb);
    if (nb.empty()) return 0;
    const float r2 = nb.back().first;
    if (!(r2 > 0)) return 0;
    float X = 0, Y = 0, Z = 0;
    for (const auto& e : nb) {
        const float* om = pm.omega_in[0] + 3 * e.second;
        if (om[0] * c.N.x + om[1] * c.N.y + om[2] * c.N.z > 0) {
            X += pm.power[0][3 * e.second];
            Y += pm.power[0][3 * e.second + 1];
            Z += pm.power[0][3 * e.second + 2];
        }
    }
    const float inv = 1.0f / (3.14159265358979323846f * r2);
    int32_t idx[3];
    float w[3];
    if (!pm_locate(pm, X * inv, Y * inv, Z * inv, idx, w)) return 0;
    return pm_recover(pm, idx, w, P.lam);
}

// traceDirect with highQuality false (direct_lighting.cpp:236-262)
float dl_direct_lq(const DLPath& P, const Bsdf& B, const Ctx& c, V wi, V start, uint32_t key) {
    const Scene& S = *P.S;
    const int nlights = (int)S.in.n_lights;
    if (nlights <= 0) return 0;
    const int n = P.R->secondary_light_samples > 0 ? P.R->secondary_light_samples : 1;
    float result = 0;
    for (int k = 0; k < n; ++k) {
        const uint32_t j0 = 16u * (uint32_t)k;
        const float uc = P.smp.get(dl_dim_branch(key, j0), false);
        int l = (int)(std::lower_bound(S.light_cdf.begin(), S.light_cdf.end(), uc) - S.light_cdf.begin());
        l = std::min(l, nlights - 1);
        const float pc = light_pdf_choice(S, l);
        if (!(pc > 0)) continue;
        const int nb = S.in.lights[l].type == L_POINT ? 0 : 1;
        auto u = [&](int kind, int, int axis) {
            return P.smp.get(dl_dim_branch(key, j0 + 1u + 2u * (uint32_t)kind + (uint32_t)axis), false);
        };
        result += estimate_light(S, B, c, wi, start, l, 1, nb, P.lam, u) / ((float)n * pc);
    }
    return result;
}

uint32_t dl_dim_final_gather(int i, int axis) { return 0x600000u + (uint32_t)i * 4u + (uint32_t)axis; }

// estimateRadiance (photon_mapper.cpp:1282-1336): from the irradiance map's nearest point within
// the global radius when there is a map, else the global map's k nearest photons; *sqr gets the
// estimate's squared radius (the radius itself, as the reference assigns it, when nothing is found;
// infinity without a diffuse part)
float pm_radiance(const DLPath& P, const Ctx& c, const Bsdf& B, V wi, float* sqr) {
    const PmIn& pm = *P.pm;
    *sqr = INFINITY;
    if (!has(B.caps, C_DIFF)) return 0;
    if (pm.n_irr > 0) {
        const float r2max = pm.radius[0] * pm.radius[0];
        int64_t best = -1;
        float bd = INFINITY;
        for (uint64_t i = 0; i < pm.n_irr; ++i) {
            const float dx = pm.irr_position[3 * i] - c.target.x, dy = pm.irr_position[3 * i + 1] - c.target.y,
                        dz = pm.irr_position[3 * i + 2] - c.target.z;
            const float d2 = dx * dx + dy * dy + dz * dz;
            if (d2 < r2max && d2 < bd) {
                bd = d2;
                best = (int64_t)i;
            }
        }
        if (best < 0) {
            *sqr = pm.radius[0];
            return 0;
        }
        *sqr = pm.irr_r2[best];
        const float* n = pm.irr_normal + 3 * best;
        const V wo{n[0] * c.u.x + n[1] * c.u.y + n[2] * c.u.z, n[0] * c.v.x + n[1] * c.v.y + n[2] * c.v.z,
                   n[0] * c.N.x + n[1] * c.N.y + n[2] * c.N.z};
        const Out be = evaluate(B, wi, wo, C_ALL);
        if (!(be.pdf > 0) || be.value == 0) return 0;
        return be.value * pm_recover(pm, pm.irr_blend_idx + 3 * best, pm.irr_blend_w + 3 * best, P.lam);
    }
    if (pm.n[0] == 0 || pm.k[0] < 1) return 0;
    thread_local std::vector<std::pair<float, int64_t>> nb;
    pm_nearest(pm, 0, c.target, nb);
    if (nb.size() < 2) {
        *sqr = pm.radius[0];
        return 0;
    }
    *sqr = nb.back().first;
    return pm_estimate(P, 0, c, B, wi);
}

float pm_gather_indirect(const DLPath& P, const Ctx& c, const Bsdf& B, V wi, V origin, int n, int stage,
                         uint32_t key);

// traceGatherRay (photon_mapper.cpp:1150-1190)
float pm_trace_gather(const DLPath& P, V o, V d, float tmin, int stage, uint32_t key) {
    const Scene& S = *P.S;
    const Hit h = oracle_internal::tree_closest(S.tree, Ray{o.x, o.y, o.z, tmin, d.x, d.y, d.z, INFINITY});
    if (h.prim < 0) return 0;
    const Ctx c = hit_ctx(S, o, d, h);
    if (c.mi < 0) return pm_trace_gather(P, o, d, h.t + TOL, stage, key);  // entering or leaving something
    const Material& M = S.in.materials[c.mi];
    if (M.type == M_NONE) return 0;
    const Bsdf B = make_bsdf(S, M, c, P.lam);
    const V md = -d;
    V wi{dot(md, c.u), dot(md, c.v), dot(md, c.N)};
    wi.z = std::max(wi.z, 1.19209290e-07f);
    float sqr;
    const float radiance = pm_radiance(P, c, B, wi, &sqr);
    if (h.t * h.t < sqr && stage == 0 && P.pm->fg_secondary > 0) {
        // gatherSecondary (:1195-1219)
        const V point = o + h.t * d;
        return pm_gather_indirect(P, c, B, wi, point, P.pm->fg_secondary, 1, key) +
               dl_direct_lq(P, B, c, wi, c.target + (10.0f * TOL) * c.N, key);
    }
    return radiance;
}

// gatherIndirect (:1060-1146): n BSDF samples of the reflective diffuse part, each traced as a
// gather ray; the first stage's samples are per-sample dimensions, the second stage's hashes of
// the ray's key
float pm_gather_indirect(const DLPath& P, const Ctx& c, const Bsdf& B, V wi, V origin, int n, int stage,
                         uint32_t key) {
    float result = 0;
    for (int i = 0; i < n; ++i) {
        float u0, u1, uc;
        uint32_t gk;
        if (stage == 0) {
            u0 = P.smp.get(dl_dim_final_gather(i, 0), true);
            u1 = P.smp.get(dl_dim_final_gather(i, 1), true);
            uc = P.smp.get(dl_dim_final_gather(i, 2), true);
            gk = dl_child_key(key, 0x200u + (uint32_t)i);
        } else {
            gk = dl_child_key(key, 0x300u + (uint32_t)i);
            u0 = P.smp.get(dl_dim_branch(gk, 0x2000u), false);
            u1 = P.smp.get(dl_dim_branch(gk, 0x2001u), false);
            uc = P.smp.get(dl_dim_branch(gk, 0x2002u), false);
        }
        const Out out = sample(B, wi, u0, u1, uc, C_REFL | C_DIFF);
        if (!out) continue;
        const V wd = out.wo.x * c.u + out.wo.y * c.v + out.wo.z * c.N;
        const float radiance = pm_trace_gather(P, origin, wd, TOL, stage, gk);
        result += radiance * (out.value * (std::fabs(out.wo.z) / ((float)n * out.pdf)));
    }
    return result;
}

float dl_cast(DLPath& P, V o, V d, float tmin, float tmax, int gen, bool hq, uint32_t key) {
    const Scene& S = *P.S;
    const RenderIn& R = *P.R;
    if (gen > R.max_ray_generation) return 0;
    const Hit h = oracle_internal::tree_closest(S.tree, Ray{o.x, o.y, o.z, tmin, d.x, d.y, d.z, tmax});
    if (h.prim < 0) {
        if (gen == 0 && S.sky >= 0 && S.sky_distance > tmin * (1 + TOL) && S.sky_distance < tmax * (1 - TOL)) P.alpha = 1;
        return 0;
    }
    if (gen == 0) P.alpha = 1;
    Ctx c = hit_ctx(S, o, d, h);
    if (gen == 0 && S.in.n_textures > 0) camera_footprint(S, R, P.smp, (uint32_t)h.prim, c);  // the camera vertex
    if (c.mi < 0) return dl_cast(P, o, d, h.t + TOL, tmax, gen + 1, hq, dl_child_key(key, 0));
    const Material& M = S.in.materials[c.mi];
    if (P.pm && P.pm->visualize) return pm_irradiance(P, c);
    float result = 0;
    if ((gen == 0 || c.light < 0) && M.emission >= 0) result += spectrum(S, M.emission, P.lam, false);
    if (M.type == M_NONE) return result;
    const Bsdf B = make_bsdf(S, M, c, P.lam);
    const V md = -d;
    V wi{dot(md, c.u), dot(md, c.v), dot(md, c.N)};
    wi.z = std::max(wi.z, 1.19209290e-07f);
    const V start = c.target + (10.0f * TOL) * c.N;
    const int nlights = (int)S.in.n_lights;
    if (P.pm && has(B.caps, C_DIFF)) {
        result += pm_estimate(P, 1, c, B, wi);  // estimateCaustics
        if (hq && P.pm->fg_rays > 0) {
            result += pm_gather_indirect(P, c, B, wi, start, P.pm->fg_rays, 0, key);
        } else {
            float sqr;
            result += pm_radiance(P, c, B, wi, &sqr);
        }
    }
    if (P.pm && !P.pm->ray_direct) {
        // no traced direct light: the global map holds it
    } else if (hq) {
        for (int l = 0; l < nlights; ++l) {
            const Light& L = S.in.lights[l];
            const int nl = L.emission_samples > 0 ? L.emission_samples : 1;
            const int nb = L.type == L_POINT ? 0 : nl;
            auto u = [&](int kind, int k, int axis) {
                const int ax = kind == 0 ? axis : (kind == 1 ? 2 + axis : 4);
                return P.smp.get(dl_dim_light(l, k, ax), true);
            };
            result += estimate_light(S, B, c, wi, start, l, nl, nb, P.lam, u);
        }
    } else {
        result += dl_direct_lq(P, B, c, wi, start, key);
    }
    // traced specular and glossy scattering
    const uint32_t glossy = R.trace_glossy < 0 ? 0u : (uint32_t)C_GLOSSY;
    const uint32_t sg = C_REFL | C_TRANS | C_SPEC | glossy;
    if (compatible(B.caps, sg) && gen + 1 <= R.max_ray_generation) {
        const int ns = hq ? (M.samples > 0 ? M.samples : 1) : 1;
        for (int side = 0; side < 2; ++side) {
            const uint32_t dir_cap = side == 0 ? C_REFL : C_TRANS;
            if (!has(B.caps, dir_cap)) continue;
            for (int i = 0; i < ns; ++i) {
                float u0, u1, uc;
                if (hq) {
                    u0 = P.smp.get(dl_dim_scatter(i, 3 * side), true);
                    u1 = P.smp.get(dl_dim_scatter(i, 3 * side + 1), true);
                    uc = P.smp.get(dl_dim_scatter(i, 3 * side + 2), true);
                } else {
                    const uint32_t j0 = 0x1000u + 8u * (uint32_t)side;
                    u0 = P.smp.get(dl_dim_branch(key, j0), false);
                    u1 = P.smp.get(dl_dim_branch(key, j0 + 1u), false);
                    uc = P.smp.get(dl_dim_branch(key, j0 + 2u), false);
                }
                const Out bs = sample(B, wi, u0, u1, uc, dir_cap | C_SPEC | glossy);
                if (!bs || (side == 0 ? !(bs.wo.z > 0) : !(bs.wo.z < 0))) continue;
                const V wd = bs.wo.x * c.u + bs.wo.y * c.v + bs.wo.z * c.N;
                const V begin = c.target + ((side == 0 ? 10.0f : -10.0f) * TOL) * c.N;
                const float child = dl_cast(P, begin, wd, TOL, INFINITY, gen + 1, hq && is_specular(B),
                                            dl_child_key(key, 2u * (uint32_t)i + (uint32_t)side));
                result += bs.value * child * (std::fabs(bs.wo.z) / ((float)ns * bs.pdf));
            }
        }
    }
    return result;
}

}  // namespace

extern "C" {

// the recovery table of image textures (copied): wavelengths, chromaticity points of the samples
// and the box corners after them, spectra, triangles
void oracle_scene_set_recovery(void* scene, const float* wavelengths, int nw, const float* points, const float* spectra,
                               int ns, const int32_t* tris, int nt) {
    Scene* S = static_cast<Scene*>(scene);
    S->rec_w.assign(wavelengths, wavelengths + nw);
    S->rec_p.assign(points, points + 2 * (size_t)(ns + 4));
    S->rec_s.assign(spectra, spectra + (size_t)ns * nw);
    S->rec_t.assign(tris, tris + 3 * (size_t)nt);
    S->rec.wavelengths = S->rec_w.data();
    S->rec.points = S->rec_p.data();
    S->rec.spectra = S->rec_s.data();
    S->rec.tris = S->rec_t.data();
    S->rec.nw = nw;
    S->rec.ns = ns;
    S->rec.nt = nt;
}

void* oracle_scene_create(const SceneIn* in) {
    Scene* S = new Scene();
    S->in = *in;
    S->tree = oracle_tree_build(in->vertices, in->n_vertices, in->triangles, in->n_triangles);
    if (in->n_spheres) oracle_tree_set_spheres(S->tree, in->spheres, in->n_spheres, in->n_triangles);
    S->spec_max.assign(in->n_spectra, 0);
    for (uint64_t k = 0; k < in->n_spectra; ++k) {
        const Spectrum& s = in->spectra[k];
        if (s.type == SP_SAMPLED) {
            float mx = -INFINITY;
            for (int i = 0; i < s.count; ++i) mx = std::max(mx, in->pool[s.offset + s.count + i]);
            S->spec_max[k] = s.p[0] > 0.0f ? s.p[0] : mx;
        }
    }
    const uint64_t nl = in->n_lights;
    S->light_cdf.assign(nl, 0);
    S->light_area.assign(nl, 0);
    S->tri_cdf.assign(in->n_triangles, 0);
    double tot = 0;
    for (uint64_t k = 0; k < nl; ++k) {
        const Light& L = in->lights[k];
        if (L.type == L_SKY) S->sky = (int)k;
        if (L.type == L_PARA) {
            const double ux = L.u[0], uy = L.u[1], uz = L.u[2], vx = L.v[0], vy = L.v[1], vz = L.v[2];
            const double cx = uy * vz - uz * vy, cy = uz * vx - ux * vz, cz = ux * vy - uy * vx;
            S->light_area[k] = (float)std::sqrt(cx * cx + cy * cy + cz * cz);
        } else if (L.type == L_MESH) {
            std::vector<double> ar(L.n_tris);
            double acc = 0;
            for (int i = 0; i < L.n_tris; ++i) {
                const uint32_t* t = in->triangles + 3 * (size_t)(L.first_tri + i);
                const float* a = in->vertices + 3 * t[0];
                const float* b = in->vertices + 3 * t[1];
                const float* c = in->vertices + 3 * t[2];
                const double e1[3] = {(double)b[0] - a[0], (double)b[1] - a[1], (double)b[2] - a[2]};
                const double e2[3] = {(double)c[0] - a[0], (double)c[1] - a[1], (double)c[2] - a[2]};
                const double nx = e1[1] * e2[2] - e1[2] * e2[1], ny = e1[2] * e2[0] - e1[0] * e2[2],
                             nz = e1[0] * e2[1] - e1[1] * e2[0];
                ar[i] = 0.5 * std::sqrt(nx * nx + ny * ny + nz * nz);
                acc += ar[i];
            }
            double run = 0;
            for (int i = 0; i < L.n_tris; ++i) {
                run += ar[i];
                S->tri_cdf[L.first_tri + i] = (float)(run / acc);
            }
            S->light_area[k] = (float)acc;
        }
        tot += std::max(0.0f, L.power);
        S->light_cdf[k] = (float)tot;
    }
    for (uint64_t k = 0; k < nl; ++k) S->light_cdf[k] = tot > 0 ? (float)(S->light_cdf[k] / tot) : (float)(k + 1) / nl;
    // observer (Observer::Observer)
    const uint64_t n = in->n_observer;
    const float* O = in->observer;
    S->ow.resize(n);
    S->oxyz.resize(3 * n);
    S->odxyz.assign(3 * n, 0);
    S->ocdf.resize(n);
    std::vector<double> dX(3 * n), cd(n, 0);
    double prev = O[0], acc = 0;
    for (uint64_t k = 0; k + 1 < n; ++k) {
        const double w = O[4 * k], wn = O[4 * (k + 1)];
        for (int c = 0; c < 3; ++c) {
            S->odxyz[3 * k + c] = (float)((O[4 * (k + 1) + 1 + c] - O[4 * k + 1 + c]) / (wn - w));
            dX[3 * k + c] = O[4 * k + 1 + c] * ((wn - prev) / 2);
        }
        prev = w;
        acc += (std::fabs(O[4 * k + 1]) + std::fabs(O[4 * k + 2]) + std::fabs(O[4 * k + 3]) + std::fabs(O[4 * (k + 1) + 1]) +
                std::fabs(O[4 * (k + 1) + 2]) + std::fabs(O[4 * (k + 1) + 3])) * (wn - w);
        cd[k + 1] = acc;
    }
    for (int c = 0; c < 3; ++c) dX[3 * (n - 1) + c] = O[4 * (n - 1) + 1 + c] * ((O[4 * (n - 1)] - prev) / 2);
    double Y = 0;
    for (uint64_t k = 0; k < n; ++k) Y += dX[3 * k + 1];
    for (uint64_t k = 0; k < n; ++k) {
        S->ow[k] = O[4 * k];
        for (int c = 0; c < 3; ++c) {
            S->oxyz[3 * k + c] = (float)(O[4 * k + 1 + c] / Y);
            S->odxyz[3 * k + c] = (float)(S->odxyz[3 * k + c] / Y);
        }
        S->ocdf[k] = (float)(cd[k] / acc);
    }
    S->ocdf[n - 1] = 1;
    S->sky_distance = in->scene_radius > 0 ? 1e3f * in->scene_radius : 1e3f;
    return S;
}

void oracle_scene_free(void* s) {
    Scene* S = static_cast<Scene*>(s);
    if (S->tree) oracle_tree_free(S->tree);
    delete S;
}

uint64_t oracle_mix64(uint64_t z) { return mix64(z); }

// ---- photon tracing: PhotonMapper::emitPhoton / tracePhoton (tracers/photon_mapper.cpp:628-796)
struct PhotonIn {
    int32_t max_ray_generation, ray_traced_direct;
    uint64_t seed, global_target, max_emitted, wave;
    int32_t final_gather;
    float caustics_quality;
};
static_assert(sizeof(PhotonIn) == sizeof(liar_photon_desc), "oracle mirror out of step with include/liar_gpu.h");
struct PhotonRec {
    float pos[3], omega[3], power[3];
    uint32_t path, tag;
};

static void trace_photon_rec(const Scene& S, const PhotonIn& D, const Sampler& smp, uint32_t path, float lam,
                             float lam_pdf, float power, V o, V d, float tmin, float tmax, int gen, bool caustic,
                             std::vector<PhotonRec>& out) {
    if (power == 0) return;
    const Hit h = oracle_internal::tree_closest(S.tree, Ray{o.x, o.y, o.z, tmin, d.x, d.y, d.z, tmax});
    if (h.prim < 0) return;
    const V hit = o + h.t * d;
    const uint32_t prim = (uint32_t)h.prim;
    const int obj = prim < S.in.n_triangles ? S.in.triangle_object[prim] : S.in.sphere_object[prim - S.in.n_triangles];
    const int mi = S.in.object_material[obj];
    if (mi < 0) {  // no shader: entering or leaving something
        if (gen >= D.max_ray_generation) return;
        return trace_photon_rec(S, D, smp, path, lam, lam_pdf, power, o, d, h.t + TOL, tmax, gen + 1, caustic, out);
    }
    if (S.in.materials[mi].type == M_NONE) return;  // a shader without a BSDF absorbs the photon
    const Material& M = S.in.materials[mi];
    if (M.type == M_LAMBERT) {
        // storage by Russian roulette with the maps' probabilities (photon_mapper.cpp:733-745,
        // 1455-1462): 1 / max(q, 1) global, q / max(q, 1) caustic; the power stays, the map builder
        // divides by the probability
        const float q = D.caustics_quality == 0 ? 1.0f : std::max(D.caustics_quality, 0.0f);
        const float pg = 1.0f / std::max(q, 1.0f), pc = q / std::max(q, 1.0f);
        const uint32_t sbase = 8 + 8 * (uint32_t)gen;
        const bool to_caustic = caustic && (pc >= 1 || !(smp.get(sbase + 4, false) > pc));
        // photon_mapper.cpp:742: with final gathering every diffuse hit is a global photon
        const bool to_global = (((gen > 0 || !D.ray_traced_direct) && !caustic) || D.final_gather) &&
                               (pg >= 1 || !(smp.get(sbase + 5, false) > pg));
        if (to_caustic || to_global) {
            PhotonRec r;
            r.pos[0] = hit.x;
            r.pos[1] = hit.y;
            r.pos[2] = hit.z;
            r.omega[0] = -d.x;
            r.omega[1] = -d.y;
            r.omega[2] = -d.z;
            const float sc = power / lam_pdf;  // Photon::Photon stores power.xyz(sample)
            const V c = observer_sensitivity(S, lam);
            r.power[0] = sc * c.x;
            r.power[1] = sc * c.y;
            r.power[2] = sc * c.z;
            r.path = path;
            r.tag = (to_caustic ? 2u : 0u) | (to_global ? 1u : 0u) | ((uint32_t)gen << 8);
            out.push_back(r);
        }
    }
    if (gen >= D.max_ray_generation) return;
    // the same local context as the path tracer
    const Ctx lc = hit_ctx(S, o, d, h);
    const bool leaving = lc.leaving;
    const V ng = lc.ng, N = lc.N, u = lc.u, v = lc.v;
    const float uv_u = lc.uv_u, uv_v = lc.uv_v;
    Bsdf B{};
    B.type = M.type;
    B.mdf = M.mdf;
    B.ng = {dot(ng, u), dot(ng, v), dot(ng, N)};
    B.eta = B.kappa = B.ior = B.etaI = B.etaT = 1;
    B.au = sq(std::max(M.rough_u, 1e-3f));
    B.av = sq(std::max(M.rough_v, 1e-3f));
    switch (M.type) {
        case M_LAMBERT:
            B.caps = C_REFL | C_DIFF;
            B.r = param(S, M, 0, TexPoint{uv_u, uv_v, 0, 0, 0, 0, 0, hit}, lam, true);
            break;
        case M_CONDUCTOR:
        case M_CT:
            B.caps = M.type == M_CONDUCTOR ? (C_REFL | C_SPEC) : (C_REFL | C_GLOSSY);
            B.eta = std::max(param(S, M, 0, TexPoint{uv_u, uv_v, 0, 0, 0, 0, 0, hit}, lam, false), 1e-9f);
            B.kappa = std::max(param(S, M, 1, TexPoint{uv_u, uv_v, 0, 0, 0, 0, 0, hit}, lam, false), 1e-9f);
            B.r = param(S, M, 2, TexPoint{uv_u, uv_v, 0, 0, 0, 0, 0, hit}, lam, true);
            break;
        case M_DIELECTRIC: {
            B.caps = C_REFL | C_TRANS | C_SPEC;
            const float i1 = std::max(param(S, M, 1, TexPoint{uv_u, uv_v, 0, 0, 0, 0, 0, hit}, lam, false), 1e-9f);
            const float i2 = std::max(param(S, M, 0, TexPoint{uv_u, uv_v, 0, 0, 0, 0, 0, hit}, lam, false), 1e-9f);
            B.ior = leaving ? i2 / i1 : i1 / i2;
            B.r = param(S, M, 2, TexPoint{uv_u, uv_v, 0, 0, 0, 0, 0, hit}, lam, true);
            B.t = param(S, M, 3, TexPoint{uv_u, uv_v, 0, 0, 0, 0, 0, hit}, lam, true);
            break;
        }
        case M_WALTER: {
            B.caps = C_TRANS | C_GLOSSY;
            float ei = std::max(param(S, M, 1, TexPoint{uv_u, uv_v, 0, 0, 0, 0, 0, hit}, lam, false), 1e-9f);
            float et = std::max(param(S, M, 0, TexPoint{uv_u, uv_v, 0, 0, 0, 0, 0, hit}, lam, false), 1e-9f);
            if (leaving) std::swap(ei, et);
            B.etaI = ei;
            B.etaT = et;
            B.r = param(S, M, 2, TexPoint{uv_u, uv_v, 0, 0, 0, 0, 0, hit}, lam, true);
            B.t = param(S, M, 3, TexPoint{uv_u, uv_v, 0, 0, 0, 0, 0, hit}, lam, true);
            break;
        }
        case M_MIRROR:
            B.caps = C_REFL | C_SPEC;
            B.r = param(S, M, 0, TexPoint{uv_u, uv_v, 0, 0, 0, 0, 0, hit}, lam, true);
            break;
    }
    const V md = -d;
    V wi{dot(md, u), dot(md, v), dot(md, N)};
    wi.z = std::max(wi.z, 1.19209290e-07f);
    const uint32_t base = 8 + 8 * (uint32_t)gen;
    const Out so = sample(B, wi, smp.get(base + 0, false), smp.get(base + 1, false), smp.get(base + 2, false), C_ALL);
    if (!so) return;
    const float ct = so.wo.z;
    float np = power * so.value * (std::fabs(ct) / so.pdf);
    const float prob = std::min(1.0f, np / power);
    const float ur = smp.get(base + 3, false);
    if (prob <= 0 || ur > prob) return;  // russianRoulette (kernel/kernel_common.h:160-168)
    np /= std::min(prob, 1.0f);
    const V nd = so.wo.x * u + so.wo.y * v + so.wo.z * N;
    const V start = hit + ((ct > 0 ? 10.0f : -10.0f) * TOL) * ng;
    const bool specular = M.type != M_LAMBERT;
    trace_photon_rec(S, D, smp, path, lam, lam_pdf, np, start, nd, TOL, INFINITY, gen + 1,
                     specular && (caustic || gen == 0), out);
}

static void emit_photon(const Scene& S, const PhotonIn& D, uint64_t seed, uint64_t path, std::vector<PhotonRec>& out) {
    const Sampler smp{seed, (uint32_t)path, (uint32_t)(path >> 32), 1};
    float lpdf;
    const float lam = observer_sample(S, smp.get(5, false), lpdf);
    const float ul = smp.get(0, false);
    int k = (int)(std::lower_bound(S.light_cdf.begin(), S.light_cdf.end(), ul) - S.light_cdf.begin());
    k = std::min(k, (int)S.in.n_lights - 1);
    const float pc = light_pdf_choice(S, k);
    const Light& L = S.in.lights[k];
    const float ax = smp.get(1, false), ay = smp.get(2, false), bx = smp.get(3, false), by = smp.get(4, false);
    V origin{0, 0, 0}, dir{0, 0, 1};
    float pdf = 0, value = 0;
    if (L.type == L_POINT) {
        dir = uniform_sphere(ax, ay, pdf);
        origin = {L.pos[0], L.pos[1], L.pos[2]};
        value = spectrum(S, L.spectrum, lam, false);
    } else if (L.type == L_PARA) {
        const V u{L.u[0], L.u[1], L.u[2]}, v{L.v[0], L.v[1], L.v[2]};
        origin = V{L.pos[0], L.pos[1], L.pos[2]} + ax * u + ay * v;
        V n = unit(cross(u, v));
        if (L.double_sided && 2 * bx >= 1) n = -n;
        const V a = std::fabs(n.x) > std::fabs(n.y) ? V{-n.z, 0, n.x} : V{0, n.z, -n.y};
        const V tu = unit(a), tv = cross(n, tu);
        float dpdf;
        const V ld = cosine_hemisphere(bx, by, dpdf);
        dir = ld.x * tu + ld.y * tv + ld.z * n;
        pdf = (1 / S.light_area[k]) * dpdf;
        value = spectrum(S, L.spectrum, lam, false) * ld.z;
    }
    if (!(pdf > 0 && value != 0 && pc > 0 && lpdf > 0)) return;
    trace_photon_rec(S, D, smp, (uint32_t)path, lam, lpdf, value / (pc * pdf), origin, dir, TOL, INFINITY, 0, false,
                     out);
}

// photons of the whole emission, sorted by (path, bounce); counts = stored, global, caustic, emitted
int oracle_photon_trace(void* s, const PhotonIn* D, PhotonRec* out, uint64_t capacity, uint64_t* counts, int threads) {
    const Scene& S = *static_cast<Scene*>(s);
    if (S.in.n_lights == 0) {
        counts[0] = counts[1] = counts[2] = counts[3] = 0;
        return 0;
    }
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    const uint64_t seed = mix64(D->seed ^ 0x9a1d37c8e15b22f3ull);
    const uint64_t wave = D->wave ? D->wave : (1ull << 21);
    uint64_t emitted = 0, global = 0, caustic = 0, stored = 0;
    while (emitted < D->max_emitted && global < D->global_target) {
        const uint64_t n = std::min(wave, D->max_emitted - emitted);
        std::vector<std::vector<PhotonRec>> parts(threads);
        std::atomic<uint64_t> next{0};
        auto work = [&](int t) {
            while (true) {
                const uint64_t b = next.fetch_add(1024);
                if (b >= n) break;
                for (uint64_t i = b; i < std::min(n, b + 1024); ++i) emit_photon(S, *D, seed, emitted + i, parts[t]);
            }
        };
        std::vector<std::thread> pool;
        for (int t = 1; t < threads; ++t) pool.emplace_back(work, t);
        work(0);
        for (auto& t : pool) t.join();
        std::vector<PhotonRec> all;
        for (auto& p : parts) all.insert(all.end(), p.begin(), p.end());
        std::sort(all.begin(), all.end(), [](const PhotonRec& a, const PhotonRec& b) {
            return a.path < b.path || (a.path == b.path && (a.tag >> 8) < (b.tag >> 8));
        });
        for (const PhotonRec& r : all) {
            if (stored < capacity) out[stored] = r;
            ++stored;
            if (r.tag & 1u) ++global;
            if (r.tag & 2u) ++caustic;
        }
        emitted += n;
    }
    counts[0] = stored;
    counts[1] = global;
    counts[2] = caustic;
    counts[3] = emitted;
    return stored > capacity ? -4 : 0;
}

// spectrum idx of the scene at wavelength w (Spectral Single-mode look-up)
float oracle_spectrum_eval(void* s, int idx, float w, int reflectant) {
    return spectrum(*static_cast<Scene*>(s), idx, w, reflectant != 0);
}

// Observer::sample and ::sensitivity of the scene's observer table
float oracle_observer_sample(void* s, float u, float* pdf, float* xyz) {
    const Scene& S = *static_cast<Scene*>(s);
    const float w = observer_sample(S, u, *pdf);
    const V c = observer_sensitivity(S, w);
    xyz[0] = c.x;
    xyz[1] = c.y;
    xyz[2] = c.z;
    return w;
}

// ---- the film: Raster::doWriteRender (output/raster.cpp:547-606) behind FilterTriangle
// (output/filter_triangle.cpp:100-145, kernel :167-170) or FilterMitchell
// (output/filter_mitchell.cpp:84-146): the pixel at offset (i, j) from the sample's pixel gets
// weight k(dx + i) k(dy + j), (dx, dy) the sample's offset from its pixel centre; pixels outside
// the image are dropped; a sample brighter than maxSampleLuminance in Y is scaled down to it.
static float mitchell_kernel(float x, float B) {
    const float C = (1.0f - B) / 2.0f;
    x = std::fabs(x);
    if (x < 1.0f)
        return ((12.0f - 9.0f * B - 6.0f * C) * (x * x * x) + (-18.0f + 12.0f * B + 6.0f * C) * (x * x) + (6.0f - 2.0f * B)) / 6.0f;
    if (x < 2.0f)
        return ((-B - 6.0f * C) * (x * x * x) + (6.0f * B + 30.0f * C) * (x * x) + (-12.0f * B - 48.0f * C) * x +
                (8.0f * B + 24.0f * C)) / 6.0f;
    return 0.0f;
}

static void film_add(float* f, float X, float Y, float Z, float alpha, float w) {
    const float wa = w * alpha;
    f[0] += wa * X;
    f[1] += wa * Y;
    f[2] += wa * Z;
    f[3] += wa;
    f[4] += w * (X * X);
    f[5] += w * (Y * Y);
    f[6] += w * (Z * Z);
    f[7] += w;
}

static void film_splat(const RenderIn& R, float* film, int px, int py, float jx, float jy, float X, float Y, float Z,
                       float alpha) {
    if (R.max_sample_luminance > 0.0f && Y > R.max_sample_luminance) {
        const float s = R.max_sample_luminance / Y;
        X *= s;
        Y *= s;
        Z *= s;
    }
    if (R.filter == 0) {
        film_add(film + 8 * ((int64_t)py * R.width + px), X, Y, Z, alpha, 1.0f);
        return;
    }
    const bool mitchell = R.filter == 2;
    const float param = mitchell ? (R.filter_param != 0.0f ? R.filter_param : 1.0f / 3.0f)
                                 : (R.filter_param > 0.0f ? R.filter_param : 1.0f);
    const int r = mitchell ? 2 : (int)std::ceil(param);
    const float dx = jx - 0.5f, dy = jy - 0.5f;
    for (int j = -r; j <= r; ++j) {
        const int y = py + j;
        if (y < 0 || y >= R.height) continue;
        const float fy = mitchell ? mitchell_kernel(dy + (float)j, param) : std::max(0.0f, param - std::fabs(dy + (float)j));
        for (int i = -r; i <= r; ++i) {
            const int x = px + i;
            if (x < 0 || x >= R.width) continue;
            const float fx = mitchell ? mitchell_kernel(dx + (float)i, param) : std::max(0.0f, param - std::fabs(dx + (float)i));
            film_add(film + 8 * ((int64_t)y * R.width + x), X, Y, Z, alpha, fx * fy);
        }
    }
}

int render_body(void* s, const RenderIn* R, const PmIn* pm, float* film, int64_t pixel_begin, int64_t pixel_end,
                int threads);

// renders pixels [pixel_begin, pixel_end) of the image into film (8 floats per pixel, summed)
int oracle_render(void* s, const RenderIn* R, float* film, int64_t pixel_begin, int64_t pixel_end, int threads) {
    return render_body(s, R, nullptr, film, pixel_begin, pixel_end, threads);
}

// the PhotonMapper (tracer 2) with the given maps
int oracle_render_pm(void* s, const RenderIn* R, const PmIn* pm, float* film, int64_t pixel_begin, int64_t pixel_end,
                     int threads) {
    if (!pm) return -1;
    return render_body(s, R, pm, film, pixel_begin, pixel_end, threads);
}

int render_body(void* s, const RenderIn* R, const PmIn* pm, float* film, int64_t pixel_begin, int64_t pixel_end,
                int threads) {
    const Scene& S = *static_cast<Scene*>(s);
    const int64_t npix = (int64_t)R->width * R->height;
    if (pixel_end < 0 || pixel_end > npix) pixel_end = npix;
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    const uint64_t seed = mix64(R->seed ^ mix64(0x51ed270b27ad0e0dull + (uint64_t)(uint32_t)R->first_sample));
    std::atomic<int64_t> next{pixel_begin};
    // with a filter, a sample reaches its neighbours' pixels too: every thread sums into a film of
    // its own, added to the caller's at the end
    std::vector<std::vector<float>> own(R->filter != 0 ? (size_t)threads : 0);
    std::atomic<int> slot{0};
    auto work = [&]() {
        float* target = film;
        if (R->filter != 0) {
            auto& v = own[(size_t)slot.fetch_add(1)];
            v.assign((size_t)npix * 8, 0.0f);
            target = v.data();
        }
        while (true) {
            const int64_t px = next.fetch_add(1);
            if (px >= pixel_end) break;
            for (int smp = 0; smp < R->spp; ++smp) {
                Path P;
                P.S = &S;
                P.R = R;
                P.smp = Sampler{seed, (uint32_t)px, (uint32_t)smp, (uint32_t)R->spp, (uint32_t)R->sampler};
                const uint32_t ix = (uint32_t)(px % R->width), iy = (uint32_t)(px / R->width);
                float jx, jy;
                P.smp.get2(D_SCREEN, jx, jy);
                float lpdf;
                P.lam = observer_sample(S, P.smp.get(D_LAMBDA, true), lpdf);
                const Camera& C = R->camera;
                float sx, sy, lu, lv, factor;
                camera_samples(*R, P.smp, sx, sy, lu, lv);
                V pos, dir;
                camera_at(C, sx, sy, lu, lv, pos, dir, factor);
                float L;
                if (R->tracer == 1 || R->tracer == 2) {
                    DLPath D{&S, R, P.smp, P.lam};
                    D.pm = R->tracer == 2 ? pm : nullptr;
                    L = dl_cast(D, pos, dir, std::max(TOL, factor * C.near_limit), factor * C.far_limit, 0, true, 1u);
                    P.alpha = D.alpha;
                } else {
                    L = trace_photon(P, pos, dir, std::max(TOL, factor * C.near_limit), factor * C.far_limit, 0);
                }
                float X = 0, Yv = 0, Z = 0;
                if (lpdf > 0) {
                    const float sc = L / lpdf;
                    const V c = observer_sensitivity(S, P.lam);
                    X = sc * c.x;
                    Yv = sc * c.y;
                    Z = sc * c.z;
                }
                film_splat(*R, target, (int)ix, (int)iy, jx, jy, X, Yv, Z, P.alpha);
            }
        }
    };
    std::vector<std::thread> pool;
    for (int k = 1; k < threads; ++k) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    for (const auto& v : own)
        for (size_t k = 0; k < v.size(); ++k) film[k] += v[k];
    return 0;
}

}  // extern "C"
