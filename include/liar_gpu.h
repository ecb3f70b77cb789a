/* liar_gpu.h -- C ABI of the B200 (sm_100a) implementation of LiAR's per-sample hot path.
 *
 * Conventions
 *   - Every function returns LIAR_OK (0) or a negative LIAR_ERR_* code and never throws.
 *     liar_gpu_last_error(ctx) returns a readable message for the last failure on ctx.
 *   - The caller owns every host buffer it passes. The library owns the device memory behind
 *     the opaque handles (liar_gpu_ctx, liar_gpu_mesh, ...), released by the matching
 *     *_destroy call.
 *   - A context is bound to one CUDA device and is not re-entrant: use one context per host
 *     thread. It replaces the reference's per-worker clone of tracer and sampler
 *     (src/liar/kernel/render_engine.cpp:317-326).
 *   - Functions without a "_device" suffix take HOST buffers and block until the result is
 *     back in host memory. "_device" variants take device pointers and a cudaStream_t (passed
 *     as void*, NULL = the context's stream) and return without synchronising.
 *   - "_device" calls of one context share its device scratch (work counters, status word,
 *     reorder buffers): give them one stream, or order their streams with events. The photon
 *     gather additionally orders itself after the previous gather of the same context, whatever
 *     the streams, because its reorder buffer decides where results are written.
 */
#ifndef LIAR_GPU_H
#define LIAR_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LIAR_GPU_ABI_VERSION 1

enum liar_status {
    LIAR_OK = 0,
    LIAR_ERR_INVALID = -1,     /* bad argument: null pointer, size, index out of range, NaN */
    LIAR_ERR_CUDA = -2,        /* a CUDA runtime call failed */
    LIAR_ERR_NO_DEVICE = -3,   /* no CUDA device, or the device is not sm_100 */
    LIAR_ERR_OOM = -4,         /* device or host allocation failed */
    LIAR_ERR_STACK = -5,       /* a traversal stack overflowed (tree deeper than the stack) */
    LIAR_ERR_TIMEOUT = -6,     /* a bounded device-side wait gave up */
    LIAR_ERR_CANCELLED = -7,   /* the host-mapped cancel flag was raised */
    LIAR_ERR_UNSUPPORTED = -8  /* feature combination not implemented */
};

typedef struct liar_gpu_ctx liar_gpu_ctx;
typedef struct liar_gpu_mesh liar_gpu_mesh;

/* A ray with its parameter interval, 32 bytes: the BoundedRay of the reference
 * (src/liar/kernel/bounded_ray.h:41-90). Direction need not be normalised; t is measured in
 * units of |d|. */
typedef struct liar_ray {
    float ox, oy, oz, tmin;
    float dx, dy, dz, tmax;
} liar_ray;

/* Result of one ray, 8 bytes. prim is the index of the triangle in the caller's triangle array
 * (the reference's Intersection special field k, src/liar/scenery/triangle_mesh.cpp:309), or
 * -1 on a miss. For any-hit queries prim is some occluding triangle and t its distance. */
typedef struct liar_hit {
    int32_t prim;
    float t;
} liar_hit;

/* Options of the 4-wide SAH tree build. Zero-initialised options select the defaults. */
typedef struct liar_build_opts {
    int max_leaf_size;   /* triangles per leaf, 1..8 (default 4) */
    int sah_bins;        /* 0 = full sweep SAH; else binned SAH with this many bins (default 0) */
    float traversal_cost;/* SAH cost of one node visit relative to one triangle test (default 1.0) */
    int threads;         /* host threads for the build, 0 = all cores */
} liar_build_opts;

typedef struct liar_mesh_stats {
    uint64_t n_triangles;
    uint64_t n_nodes;        /* 4-wide inner nodes, 128 bytes each */
    uint64_t n_leaves;
    uint32_t max_depth;      /* inner-node levels from the root to the deepest leaf */
    uint32_t stack_needed;   /* traversal stack entries the deepest path can need */
    double sah_cost;         /* SAH cost of the 4-wide tree (node visits + triangle tests) */
    uint64_t device_bytes;   /* bytes of device memory held by the mesh */
    double build_seconds;    /* host time of the build */
} liar_mesh_stats;

/* Launch shape of the trace kernels of a context (no reference counterpart: tuning only; the
 * results do not depend on it). */
typedef struct liar_trace_config {
    int block_size;   /* threads per block: 128 or 256 */
    int smem_stack;   /* traversal stack entries per lane kept in shared memory: 8, 16 or 24
                         (256-thread blocks: 8 or 16); deeper entries spill to local memory */
} liar_trace_config;

/* ---- context ------------------------------------------------------------------------------ */

int liar_gpu_create(liar_gpu_ctx** out, int device);
void liar_gpu_destroy(liar_gpu_ctx* ctx);
const char* liar_gpu_last_error(const liar_gpu_ctx* ctx);
int liar_gpu_abi_version(void);
/* The stream used by the host-buffer entry points and by "_device" calls given stream NULL.
 * NULL here selects the context's own non-blocking stream. */
int liar_gpu_set_stream(liar_gpu_ctx* ctx, void* stream);
/* Waits for the context's stream and reports device-side errors of the "_device" calls
 * queued since the last check (stack overflow, bounded-wait timeout, cancel). */
int liar_gpu_synchronize(liar_gpu_ctx* ctx);
/* Cancellation, the counterpart of RenderEngine::isCanceling (src/liar/kernel/render_engine.cpp:
 * 239-242, 294-297, 342): the renders of ctx read *flag between waves and bounces and, once it is
 * non-zero, queue no more work, wait for the work in flight and return LIAR_ERR_CANCELLED. The film
 * then holds the samples of the paths that finished (a partial image, like the reference's
 * cancelled render, not an estimate to keep). flag is the caller's host memory (any thread may
 * set it) and must stay valid until it is replaced; NULL removes it. */
int liar_gpu_set_cancel_flag(liar_gpu_ctx* ctx, const volatile int32_t* flag);
/* Failure injection for tests of the device-side timeout path (no reference counterpart). With
 * LIAR_FAULT_TEST_GUIDE_WAIT the guide network kernels of ctx issue no tensor-core work and wait,
 * with a short limit, for a completion that nothing signals: every such launch records a timeout,
 * frees its tensor memory and returns, and the next liar_gpu_synchronize reports
 * LIAR_ERR_TIMEOUT with the context still usable. 0 turns it off. */
enum liar_fault_test { LIAR_FAULT_TEST_NONE = 0, LIAR_FAULT_TEST_GUIDE_WAIT = 1 };
int liar_gpu_set_fault_test(liar_gpu_ctx* ctx, int mode);
/* Selects / reads the trace kernels' launch shape (default 128 threads, 16 shared entries). */
int liar_gpu_set_trace_config(liar_gpu_ctx* ctx, const liar_trace_config* cfg);
int liar_gpu_get_trace_config(const liar_gpu_ctx* ctx, liar_trace_config* out);

/* ---- triangle mesh: build + closest/any hit -----------------------------------------------
 * Replaces TriangleMesh::TriangleMesh with its Lass QbvhTree<..., SAHSplitHeuristics> reset
 * (src/liar/scenery/triangle_mesh.cpp:69-85, src/liar/scenery/triangle_mesh.h:53) and
 * ObjectTree::doPreProcess (src/liar/scenery/object_trees.h:100-108). */
int liar_gpu_mesh_build(liar_gpu_ctx* ctx, const float* vertices /* n_vertices x 3 */, size_t n_vertices,
                        const uint32_t* triangles /* n_triangles x 3 vertex indices */, size_t n_triangles,
                        const liar_build_opts* opts /* NULL = defaults */, liar_gpu_mesh** out);
void liar_gpu_mesh_destroy(liar_gpu_mesh* mesh);
int liar_gpu_mesh_stats(const liar_gpu_mesh* mesh, liar_mesh_stats* out);

/* Closest hit (any_hit = 0) replaces TriangleMesh::doIntersect
 * (src/liar/scenery/triangle_mesh.cpp:291-318): the nearest t > tmin, then accepted only if
 * BoundedRay::inRange holds, t > tmin*(1+tol) && t < tmax*(1-tol) with tol = 1e-6
 * (src/liar/kernel/bounded_ray.h:69-77, src/liar/kernel/kernel_common.cpp:32). Equal t is
 * resolved to the lower triangle index.
 * Any hit (any_hit = 1) replaces TriangleMesh::doIsIntersecting
 * (src/liar/scenery/triangle_mesh.cpp:321-330): is there a triangle with tmin < t < tmax. */
int liar_gpu_trace(liar_gpu_ctx* ctx, const liar_gpu_mesh* mesh, const liar_ray* rays, size_t n_rays,
                   liar_hit* hits, int any_hit);
int liar_gpu_trace_device(liar_gpu_ctx* ctx, const liar_gpu_mesh* mesh, const liar_ray* d_rays, size_t n_rays,
                          liar_hit* d_hits, int any_hit, void* stream);
/* Same as liar_gpu_trace_device, and adds per-ray node visits and triangle tests into
 * d_counters[0] and d_counters[1] (two uint64 on the device, accumulated). */
int liar_gpu_trace_counted_device(liar_gpu_ctx* ctx, const liar_gpu_mesh* mesh, const liar_ray* d_rays,
                                  size_t n_rays, liar_hit* d_hits, int any_hit, unsigned long long* d_counters,
                                  void* stream);

/* ---- spectral path tracing ------------------------------------------------------------------
 * A flattened scene: one triangle soup (parallelograms arrive as two triangles, meshes as their
 * triangles) whose triangles carry an object index; objects carry a material and a light. */

typedef struct liar_gpu_scene liar_gpu_scene;

/* Spectrum evaluated at one wavelength (metres), the reference's Spectral `Single` mode
 * (src/liar/kernel/spectral.cpp:178-220). */
enum liar_spectrum_type {
    LIAR_SPEC_CONSTANT = 0,  /* p[0] */
    LIAR_SPEC_SAMPLED = 1,   /* piecewise linear: pool[offset .. +count) wavelengths, then count values
                                (spectra/sampled.cpp:128, kernel/spectral.cpp:185-210); as a reflectance
                                divided by its maximum when above 1, or by p[0] when p[0] > 0 (a colour
                                recovered from XYZ, spectra/recovery_meng_simon.cpp:151-166) */
    LIAR_SPEC_BLACKBODY = 2, /* p[0] temperature (K), p[1] scale; normalised at the peak (spectra/black_body.cpp:55-118) */
    LIAR_SPEC_CAUCHY = 3     /* p[0] + p[1] / lambda_um^2 (spectra/cauchy.cpp:72-76) */
};
typedef struct liar_spectrum {
    int32_t type, offset, count;
    float p[3];
} liar_spectrum;

/* Shaders (src/liar/shaders/). spec[] holds spectrum indices (-1 = absent):
 *   LAMBERT        spec[0] diffuse                                   (lambert.cpp:105-124)
 *   CONDUCTOR      spec[0] eta, spec[1] kappa, spec[2] reflectance   (conductor.cpp:179-196)
 *   COOK_TORRANCE  spec[0] eta, spec[1] kappa, spec[2] reflectance, rough_u/v, mdf (cook_torrance.cpp:189-295)
 *   DIELECTRIC     spec[0] inner ior, spec[1] outer ior, spec[2] reflectance, spec[3] transmittance (dielectric.cpp:148-245)
 *   WALTER         as DIELECTRIC plus rough_u/v, mdf                   (walter.cpp:215-415)
 *   MIRROR         spec[0] reflectance                                 (mirror.cpp)
 *   NONE           no BSDF: rays pass through (AdjointPhotonTracer's null-shader branch)
 * emission: spectrum of an Unshaded component (shaders/unshaded.cpp:77), -1 if none. */
enum liar_material_type {
    LIAR_MAT_NONE = 0, LIAR_MAT_LAMBERT = 1, LIAR_MAT_CONDUCTOR = 2, LIAR_MAT_COOK_TORRANCE = 3,
    LIAR_MAT_DIELECTRIC = 4, LIAR_MAT_WALTER = 5, LIAR_MAT_MIRROR = 6
};
enum liar_mdf_type { LIAR_MDF_BECKMANN = 0, LIAR_MDF_GGX = 1 };
typedef struct liar_material {
    int32_t type, mdf;
    int32_t spec[4];
    int32_t emission;
    float rough_u, rough_v;
    int32_t samples;   /* DirectLighting: reflection (and transmission) samples per vertex, the shader's
                          numReflectionSamples (conductor.cpp:118, dielectric.cpp:134-144,
                          cook_torrance.cpp:182); 0 = 1 */
    int32_t tex[4];    /* texture of parameter spec[k] (index into the scene's textures), -1 = the constant
                          spectrum spec[k] */
} liar_material;

/* Textures of spectral material parameters (src/liar/textures/): a tree of nodes looked up at a
 * hit's (u, v) coordinates. A camera hit carries the screen-space footprint of the camera's ray
 * differentials (kernel/camera.cpp:53-60, intersection_context.cpp:295-324): the derivatives of
 * (u, v) and of the hit point; every other hit has a zero footprint.
 *   CONSTANT      spectrum                                    (textures/constant.cpp)
 *   CHECKER       a where the fractional (u, v) lie on the same side of split p[0], p[1], else b
 *                 (CheckerBoard, checker_board.cpp:113-207); p[2] = 1: bilinear anti-aliasing, the
 *                 share of a over the footprint's (u, v) box blends a and b
 *   GRID          a on the lines of half thickness p[0] (u, and v from below) and p[1] (v from
 *                 above), else b (GridBoard, grid_board.cpp:60-67)
 *   UV_TRANSFORM  child a at (p[0] u + p[1] v + p[2], p[3] u + p[4] v + p[5]) (TransformationUv)
 *   IMAGE         an a x b image of XYZ pixels (rows from the top) with its mip levels, looked up
 *                 at (u, 1 - v) with wrap-around by nearest pixel (p[0] = 0), bilinearly (p[0] = 1)
 *                 or trilinearly across levels (p[0] = 2) (Image, textures/image.cpp:249-718); the
 *                 XYZ becomes a spectrum through the context's recovery table (Spectral::fromXYZ),
 *                 so scenes with images need liar_gpu_set_recovery first. texture_pixels[pixels]
 *                 holds int32 bits {levels along u, levels along v, mip mode (0 none, 1 isotropic,
 *                 2 anisotropic), 0}; the next levels_u x levels_v entries hold {offset low 31 bits,
 *                 offset high bits, width, height} of level (iu, iv) at index iv x levels_u + iu,
 *                 its pixels at texture_pixels[pixels + offset]
 *   NOISE         Perlin noise of the hit point (p[0] = 0: Perlin, perlin.cpp:60-205) or its fractal
 *                 sum over up to p[0] octaves with falloff p[1], fewer for a wide footprint (FBm,
 *                 fbm.cpp:62-101), a flat spectrum; permutation tables: 3 x 257 bytes at `pixels`
 *                 of the scene's noise_tables
 *   ABS           |child a| (Abs, abs.cpp:26-35)
 *   AFFINE        p[0] child a + p[1], the child looked up as an illuminant and the result
 *                 clamped to 1 as a reflectance (Product / Sum with one non-constant input,
 *                 product.cpp:90-99, sum.cpp:90-105)
 * A lookup applies at most 8 ABS / AFFINE / anti-aliased CHECKER nodes along any path. */
enum liar_texture_type {
    LIAR_TEX_CONSTANT = 0, LIAR_TEX_CHECKER = 1, LIAR_TEX_GRID = 2, LIAR_TEX_UV_TRANSFORM = 3, LIAR_TEX_IMAGE = 4,
    LIAR_TEX_NOISE = 5, LIAR_TEX_ABS = 6, LIAR_TEX_AFFINE = 7
};
typedef struct liar_texture {
    int32_t type, a, b, spectrum;
    float p[6];
    int64_t pixels;
} liar_texture;

/* Lights (src/liar/scenery/light_*.cpp). AREA_PARALLELOGRAM: pos = support, u/v = sizes
 * (light_area.cpp + parallelogram.cpp); AREA_MESH: triangles [first_tri, first_tri + n_tris) of
 * the soup, area-CDF sampling (triangle_mesh.cpp:414-443); POINT: pos (light_point.cpp:160-196);
 * SKY: constant radiance at a fixed far distance (light_sky.cpp:140-363). power is the
 * light's total power used for the selection CDF (kernel/light_context.cpp:272-333). */
enum liar_light_type { LIAR_LIGHT_AREA_PARALLELOGRAM = 0, LIAR_LIGHT_AREA_MESH = 1, LIAR_LIGHT_POINT = 2, LIAR_LIGHT_SKY = 3 };
typedef struct liar_light {
    int32_t type, spectrum, object, double_sided;
    int32_t first_tri, n_tris;
    float pos[3], u[3], v[3];
    float power;
    int32_t emission_samples;  /* numberOfEmissionSamples (light_context.cpp:66-72): DirectLighting's
                                  light and BSDF samples per light per vertex; 0 = 1 */
} liar_light;

typedef struct liar_scene_desc {
    const float* vertices; size_t n_vertices;            /* n x 3 */
    const uint32_t* triangles; size_t n_triangles;       /* n x 3 */
    const int32_t* triangle_object;                      /* n: object of each triangle */
    const float* normals; size_t n_normals;              /* optional shading normals (n x 3) */
    const int32_t* triangle_normals;                     /* optional, n_triangles x 3 indices into normals */
    const int32_t* object_material; const int32_t* object_light; size_t n_objects;
    const liar_material* materials; size_t n_materials;
    const liar_spectrum* spectra; size_t n_spectra;
    const float* spectrum_pool; size_t pool_size;
    const liar_light* lights; size_t n_lights;
    const float* observer; size_t n_observer;            /* n x 4: wavelength (m), xbar, ybar, zbar */
    float scene_radius;                                  /* bounding sphere radius (sky distance) */
    const liar_texture* textures; size_t n_textures;     /* optional */
    const float* triangle_uvs;                           /* optional, n_triangles x 6: (u, v) per corner;
                                                            NULL: the barycentric coordinates of the hit */
    const float* texture_pixels; size_t n_texture_pixels; /* image textures: n x 4 (X, Y, Z, unused) */
    const uint8_t* noise_tables; size_t n_noise_tables;   /* noise textures' permutation tables (bytes) */
    /* analytic spheres (Sphere, scenery/sphere.cpp): n x 4 (centre, radius) and each one's object;
       sphere k is primitive n_triangles + k in hits. Their surface coordinates are
       (phi / 2 pi, theta / pi) of the outward normal (sphere.cpp:130-152). */
    const float* spheres; size_t n_spheres; const int32_t* sphere_object;
} liar_scene_desc;

/* PerspectiveCamera (src/liar/cameras/perspective_camera.cpp:406-434): direction/right/down are
 * the scaled vectors direction_ = focalLength * d, right_ = width * r, down_ = height * dn. */
typedef struct liar_camera {
    float position[3], direction[3], right[3], down[3];
    float direction_normal[3], right_normal[3], down_normal[3];
    float lens_radius, focus_distance, near_limit, far_limit;
} liar_camera;

/* ADJOINT_PHOTON: src/liar/tracers/adjoint_photon_tracer.cpp (unidirectional path tracing);
 * DIRECT_LIGHTING: src/liar/tracers/direct_lighting.cpp (direct light by
 * RayTracer::estimateLightContribution, kernel/ray_tracer.cpp:188-276, plus recursive specular
 * and glossy reflection/transmission up to max_ray_generation);
 * PHOTON_MAPPER: src/liar/tracers/photon_mapper.cpp (DirectLighting plus, at every vertex with a
 * diffuse part, the caustic map's Gaussian-filtered estimate and the global map's radiance
 * estimate, photon_mapper.cpp:466-518, 1282-1381; photon maps filled per render as
 * fillPhotonMaps / buildPhotonMap, :573-835; with final gathering at high-quality diffuse vertices,
 * gatherIndirect / traceGatherRay / gatherSecondary, :1060-1251, over the precomputed irradiance
 * map, :943-995) */
enum liar_tracer_type { LIAR_TRACER_ADJOINT_PHOTON = 0, LIAR_TRACER_DIRECT_LIGHTING = 1, LIAR_TRACER_PHOTON_MAPPER = 2 };

/* PhotonMapper settings (photon_mapper.cpp:108-142 defaults). Map 0 is the global map, map 1 the
 * caustic map. Photons bounce up to max_ray_generation; the seed of the photons is the render's. */
typedef struct liar_photon_mapper_desc {
    uint64_t max_photons;           /* maxNumberOfPhotons: emission stops here (0 = 10^8) */
    uint64_t global_map_size;       /* globalMapSize: emission stops once the global map holds this (0 = 10000) */
    float estimation_radius[2];     /* rMax of the estimates; 0 = automatic (buildPhotonMap, :815-833) */
    float estimation_tolerance[2];  /* of the automatic radius (0 = 0.05) */
    int32_t estimation_size[2];     /* photons per estimate, at most 64 (0 = 50) */
    int32_t ray_trace_direct;       /* isRayTracingDirect: -1 = false (direct light from the global map), else true */
    int32_t visualize;              /* isVisualizingPhotonMap: nonzero renders the global map's irradiance */
    int32_t final_gather_rays;      /* numFinalGatherRays, used with traced direct light (0 = no final gather) */
    int32_t secondary_gather_rays;  /* numSecondaryGatherRays: 0 = the reference's 1, -1 = none */
    float ratio_precomputed_irradiance; /* ratioPrecomputedIrradiance: 0 = the reference's 0.25, < 0 = none */
    float caustics_quality;         /* causticsQuality (photon_mapper.cpp:165-175, 1455-1462): 0 = the
                                       reference's 1, < 0 = 0 (no caustic photons); the storage
                                       probabilities of liar_photon_desc */
} liar_photon_mapper_desc;

typedef struct liar_render_desc {
    liar_camera camera;
    int32_t width, height, spp;
    int32_t tracer;
    int32_t max_ray_generation;  /* Russian roulette (survival 0.5) from this generation on (ray_tracer.cpp:171) */
    int32_t max_depth;           /* hard cap on generations, 0 = none */
    uint64_t seed;
    int32_t first_sample;        /* progressive rendering: index of the first sample of this pass */
    int32_t wave_paths;          /* paths in flight per wave, 0 = automatic */
    int32_t secondary_light_samples; /* DirectLighting.numberOfSecondaryLightSamples (0 = 1) */
    int32_t trace_glossy;        /* DirectLighting.traceGlossy: -1 = false, otherwise true */
    /* reconstruction filter between the tracer and the film (a RenderTarget wrapper in the
     * reference): LIAR_FILTER_BOX = the sample's own pixel with weight 1 (Raster alone),
     * LIAR_FILTER_TRIANGLE = FilterTriangle (output/filter_triangle.cpp:100-145, 169),
     * LIAR_FILTER_MITCHELL = FilterMitchell (output/filter_mitchell.cpp:84-150) */
    int32_t filter;
    float filter_param;          /* triangle: width (0 = 1); Mitchell: B (0 = 1/3) */
    float max_sample_luminance;  /* Raster.maxSampleLuminance (output/raster.cpp:572-575); 0 = no clamp */
    liar_photon_mapper_desc photon_mapper;  /* tracer PHOTON_MAPPER only */
    /* the sample pattern of the reference's sampler class: LIAR_SAMPLER_STRATIFIER (0;
     * samplers/stratifier.cpp: screen and lens samples on a sqrt(spp) x sqrt(spp) grid when spp is
     * a square) or LIAR_SAMPLER_LATIN_HYPERCUBE (samplers/latin_hypercube.cpp: every axis
     * stratified on its own), ORed with LIAR_SAMPLER_NOT_JITTERED for `jittered = False` (every
     * stratified value at its stratum's centre, samplers/stratifier.h:90) */
    int32_t sampler;
} liar_render_desc;

enum liar_filter { LIAR_FILTER_BOX = 0, LIAR_FILTER_TRIANGLE = 1, LIAR_FILTER_MITCHELL = 2 };
enum liar_sampler { LIAR_SAMPLER_STRATIFIER = 0, LIAR_SAMPLER_LATIN_HYPERCUBE = 1, LIAR_SAMPLER_NOT_JITTERED = 2 };

/* Uploads the scene (builds the triangle tree). */
int liar_gpu_scene_upload(liar_gpu_ctx* ctx, const liar_scene_desc* desc, liar_gpu_scene** out);
void liar_gpu_scene_destroy(liar_gpu_scene* scene);
/* Renders `spp` samples per pixel (AdjointPhotonTracer, src/liar/tracers/adjoint_photon_tracer.cpp:84-292,
 * driven like RenderEngine::render, src/liar/kernel/render_engine.cpp:170-358) and ADDS them to
 * film: width x height x 8 floats = sums of w a X, w a Y, w a Z, w a, w X^2, w Y^2, w Z^2 and w
 * over the samples that reach the pixel, w the filter weight (1 for the box filter) and a the
 * sample's alpha (the reference's Raster accumulation, src/liar/output/raster.cpp:547-606, before
 * division: the pixel is the first four sums over the last). */
int liar_gpu_render(liar_gpu_ctx* ctx, const liar_gpu_scene* scene, const liar_render_desc* desc, float* film);
/* Same on a device film buffer, asynchronous on `stream`. */
int liar_gpu_render_device(liar_gpu_ctx* ctx, const liar_gpu_scene* scene, const liar_render_desc* desc,
                           float* d_film, void* stream);
/* Path statistics of the last render on ctx: [0] paths, [1] path segments traced, [2] rays that hit. */
int liar_gpu_render_stats(const liar_gpu_ctx* ctx, unsigned long long* out3);

/* ---- batched rendering (no reference counterpart: the reference renders one scene per process)
 * Many scenes, resolutions and sample counts rendered by one CUDA-graph launch: a scene table,
 * the paths of all items in one index space cut into waves, and a device-side WHILE loop over the
 * waves (conditional graph node), each wave running raygen and `max_bounces` x (trace, shade) with
 * queue sizes that stay on the device. hero_wavelengths = 4 carries four wavelengths per path
 * (hero wavelength spectral sampling: the first is sampled from the observer, the others are
 * rotations of it over the observer's range, combined with the balance heuristic); secondary
 * wavelengths end at a dispersive (non-constant index) dielectric. */
typedef struct liar_gpu_batch liar_gpu_batch;
typedef struct liar_batch_item {
    const liar_gpu_scene* scene;
    liar_render_desc render;   /* tracer must be LIAR_TRACER_ADJOINT_PHOTON; wave_paths is ignored */
    float* d_film;             /* device film, width x height x 8 floats; samples are added */
} liar_batch_item;
typedef struct liar_batch_config {
    int32_t hero_wavelengths;  /* 1 or 4 */
    int32_t max_bounces;       /* bounces per wave; must be >= the items' max_depth (0 = that max_depth) */
    int32_t wave_paths;        /* paths in flight per wave, 0 = 4M */
    int32_t shade_blocks_per_sm; /* grid of the shade kernel: 4, 8 or 16 blocks of 128 per SM, 0 = 16 */
    liar_trace_config trace;   /* zero = the context's trace config */
} liar_batch_config;
int liar_gpu_batch_create(liar_gpu_ctx* ctx, const liar_batch_item* items, size_t n_items,
                          const liar_batch_config* cfg, liar_gpu_batch** out);
/* one cudaGraphLaunch on `stream` (NULL = the context's stream) renders every item */
int liar_gpu_batch_launch(liar_gpu_ctx* ctx, liar_gpu_batch* batch, void* stream);
/* after a launch has finished: [0] paths, [1] path segments traced, [2] segments that hit, [3] waves */
int liar_gpu_batch_stats(const liar_gpu_batch* batch, unsigned long long* out4);
void liar_gpu_batch_destroy(liar_gpu_batch* batch);

/* ---- learned path guiding (no reference counterpart: the reference's AdjointPhotonTracer samples
 * the BSDF and the lights only, src/liar/tracers/adjoint_photon_tracer.cpp:212-292)
 * A small MLP maps (position, shading normal, direction to the previous vertex) to a mixture of 8
 * von Mises-Fisher lobes over outgoing directions. Network: the 9 inputs (position normalised to
 * the config's box) -> sin/cos(pi 2^(f/2) x) for f = 0..11 plus the raw inputs (225 features) ->
 * 5 ReLU layers of 64 -> 40 outputs; bf16 weights, f32 accumulation, no biases. Trained online with
 * Adam on the renderer's own samples (KL divergence of the guide from the sampled integrand). */
typedef struct liar_gpu_guide liar_gpu_guide;
typedef struct liar_guide_config {
    float bounds_lo[3], bounds_hi[3]; /* position normalisation box (the scene's bounds) */
    float learning_rate;              /* Adam step size, 0 = 5e-3 */
    float guide_probability;          /* chance of sampling the guide at a diffuse/glossy vertex, [0, 1) */
    float light_probability;          /* chance of light sampling at a guided vertex (the reference's
                                         one-sample MIS uses 0.5), [0, 1); 0 = 0.5 */
    int32_t batch_records;            /* training records per Adam step, 0 = 65536 */
    int32_t steps_per_pass;           /* Adam steps after each rendered pass when training, 0 = 4 */
    uint64_t seed;                    /* weight initialisation */
} liar_guide_config;
int liar_gpu_guide_create(liar_gpu_ctx* ctx, const liar_guide_config* cfg, liar_gpu_guide** out);
void liar_gpu_guide_destroy(liar_gpu_guide* guide);
/* number of f32 parameters: W0 256x64, W1..W4 64x64, W5 64x48, row-major [in][out], concatenated
 * (rows 225..255 of W0 and columns 40..47 of W5 are padding and stay zero) */
size_t liar_gpu_guide_param_count(void);
int liar_gpu_guide_get_params(liar_gpu_ctx* ctx, const liar_gpu_guide* guide, float* host, size_t n);
/* replaces the weights and resets the optimiser state */
int liar_gpu_guide_set_params(liar_gpu_ctx* ctx, liar_gpu_guide* guide, const float* host, size_t n);
/* d_inputs: n x 9 floats (position, normal, direction); d_mixture: n x 40 floats = 8 lobes x
 * (mean x, y, z, concentration) then the 8 lobe weights */
int liar_gpu_guide_eval_device(liar_gpu_ctx* ctx, const liar_gpu_guide* guide, const float* d_inputs, size_t n,
                               float* d_mixture, void* stream);
/* One training step on n records of 13 floats: position, normal, direction to the previous vertex,
 * sampled direction, weight (integrand / sampling density, >= 0). apply = 0 computes the gradient
 * only. d_grad (optional) receives the gradient (param_count floats), d_loss (optional) the loss. */
int liar_gpu_guide_train_device(liar_gpu_ctx* ctx, liar_gpu_guide* guide, const float* d_records, size_t n, int apply,
                                float* d_grad, float* d_loss, void* stream);
/* draws one direction per mixture (d_mixture n x 40 as above) from uniforms d_u (n x 3: lobe
 * choice, cosine, azimuth) -> d_dirs (n x 3), d_pdf (n): the mixture density there */
int liar_gpu_guide_sample_device(liar_gpu_ctx* ctx, const float* d_mixture, const float* d_u, size_t n, float* d_dirs,
                                 float* d_pdf, void* stream);
/* [0] Adam steps taken, [1] training records produced by guided renders, [2] guided vertices,
 * [3] passes rendered */
int liar_gpu_guide_stats(const liar_gpu_guide* guide, unsigned long long* out4);
/* The AdjointPhotonTracer estimator with the guide as a third sampling technique: at a diffuse or
 * glossy vertex the directional strategy draws from the guide with probability guide_probability,
 * else from the BSDF (one-sample MIS of the mixed density against light sampling). Renders the
 * desc's spp as passes of one sample per pixel; with train != 0 every pass records (vertex,
 * direction, integrand / density) and takes steps_per_pass Adam steps before the next pass. */
int liar_gpu_render_guided_device(liar_gpu_ctx* ctx, const liar_gpu_scene* scene, liar_gpu_guide* guide,
                                  const liar_render_desc* desc, int train, float* d_film, void* stream);
/* statistics of the last guided render on ctx: [0] paths, [1] path segments, [2] segments that
 * hit, [3] directions drawn from the guide */
int liar_gpu_render_guided_stats(const liar_gpu_ctx* ctx, unsigned long long* out4);

/* ---- spectra of tristimulus values ------------------------------------------------------------
 * The context's standard recovery, as the reference's liar.Recovery.setStandard with a
 * RecoveryMengSimon (src/liar/__init__.py:72-79, spectra/recovery_meng_simon.cpp:93-310): spectra
 * (n_samples x n_wavelengths, wavelengths in metres, increasing) sampled at chromaticities xy
 * (n_samples x 2, inside [-0.3, 1.0] x [-0.3, 1.2]), and the Delaunay triangulation of those
 * points followed by the box corners (-0.3, -0.3), (1.0, -0.3), (1.0, 1.2), (-0.3, 1.2) as point
 * indices n_samples .. n_samples + 3 (n_triangles x 3). The PhotonMapper needs it (photon powers
 * are XYZ, Spectral::fromXYZ); liar_b200 sets the reference's table on every context it renders
 * with. A colour is the barycentric blend of the spectra at its triangle's corners (zero at the
 * box corners), the weights scaled to sum to X + Y + Z. Image textures need it too. A table
 * replaced by a later call stays allocated until the context is destroyed: scenes uploaded and
 * photon maps built with it keep using it. */
int liar_gpu_set_recovery(liar_gpu_ctx* ctx, const float* wavelengths, int n_wavelengths, const float* xy,
                          const float* spectra, int n_samples, const int32_t* triangles, int n_triangles);
/* The blend of each of n XYZ colours (d_xyz: n x 3): sample indices (n x 3, -1 = none) and weights
 * (n x 3); colours without a recovery get -1 and 0. */
int liar_gpu_recovery_locate_device(liar_gpu_ctx* ctx, const float* d_xyz, size_t n, int32_t* d_idx,
                                    float* d_weights, void* stream);

/* ---- photon maps -------------------------------------------------------------------------------
 * Replace the Lass KdTree<Photon> of PhotonMapper::buildPhotonMap (src/liar/tracers/photon_mapper.cpp:798-835)
 * and its rangeSearch(point, maxRadius, maxCount) (photon_mapper.cpp:1097,1257,1312,1352): for each
 * query point the (at most) k photons nearest to it with squared distance < r_max^2, in ascending
 * distance (ties: lower photon index first). Photon positions are n x 3 floats. */
typedef struct liar_gpu_photon_map liar_gpu_photon_map;
int liar_gpu_photon_map_build(liar_gpu_ctx* ctx, const float* positions, size_t n, float r_max,
                              liar_gpu_photon_map** out);
int liar_gpu_photon_map_build_device(liar_gpu_ctx* ctx, const float* d_positions, size_t n, float r_max,
                                     liar_gpu_photon_map** out, void* stream);
/* The same into an existing map (buildPhotonMap runs once per PhotonMapper::doPreProcess): its
 * device buffers are kept and grown only when the new photons need more. */
int liar_gpu_photon_map_rebuild_device(liar_gpu_ctx* ctx, liar_gpu_photon_map* map, const float* d_positions, size_t n,
                                       float r_max, void* stream);
void liar_gpu_photon_map_destroy(liar_gpu_photon_map* map);
/* idx / d2: n_queries x k (unused slots: -1 / +inf); count (optional): neighbours found. k <= 64. */
int liar_gpu_photon_gather(liar_gpu_ctx* ctx, const liar_gpu_photon_map* map, const float* queries, size_t n_queries,
                           int k, int32_t* idx, float* d2, int32_t* count);
int liar_gpu_photon_gather_device(liar_gpu_ctx* ctx, const liar_gpu_photon_map* map, const float* d_queries,
                                  size_t n_queries, int k, int32_t* d_idx, float* d_d2, int32_t* d_count, void* stream);

/* PhotonMapper::estimateIrradianceImpl (src/liar/tracers/photon_mapper.cpp:1254-1279) over gather
 * results: per query the XYZ power of the neighbours with omega_in . normal > 0, times
 * power_scale (1 / photons emitted), over pi r^2 with r^2 the farthest neighbour's d2.
 * d_power / d_omega_in: n_photons x 3; d_normals, d_out: n_queries x 3. */
int liar_gpu_photon_estimate_device(liar_gpu_ctx* ctx, const float* d_power, const float* d_omega_in, size_t n_photons,
                                    const float* d_normals, size_t n_queries, int k, const int32_t* d_idx,
                                    const float* d_d2, const int32_t* d_count, float power_scale, float* d_out,
                                    void* stream);

/* ---- photon tracing ------------------------------------------------------------------------------
 * PhotonMapper::fillPhotonMaps / emitPhoton / tracePhoton (src/liar/tracers/photon_mapper.cpp:573-796):
 * photons leave the scene's lights (chosen by power), carry power at one wavelength, scatter by
 * BSDF sampling with power-preserving Russian roulette (kernel/kernel_common.h:160) and are stored at
 * hits on surfaces with a diffuse BSDF: into the caustic map when every bounce so far was specular
 * or glossy, into the global map when not caustic and not a direct hit (isRayTracingDirect), or
 * always with final gathering (photon_mapper.cpp:742); one record per stored hit, tagged with
 * every map it belongs to.
 * Photons are emitted in waves of `wave` until the global map holds `global_target` photons or
 * `max_emitted` photons have left the lights. Stored power is XYZ (the reference's Photon record),
 * not yet divided by the number emitted. */
enum liar_photon_map_kind { LIAR_PHOTON_GLOBAL = 1, LIAR_PHOTON_CAUSTIC = 2 };
typedef struct liar_photon_desc {
    int32_t max_ray_generation;  /* photon bounces (reference default 8) */
    int32_t ray_traced_direct;   /* 1: direct photons are not stored in the global map */
    uint64_t seed;
    uint64_t global_target;      /* globalMapSize */
    uint64_t max_emitted;        /* maxNumberOfPhotons */
    uint64_t wave;               /* photons emitted per wave, 0 = automatic */
    int32_t final_gather;        /* 1: every diffuse hit goes to the global map (hasFinalGather) */
    /* causticsQuality q (0 = the reference's 1, < 0 = 0): a diffuse hit enters the global map with
     * probability 1 / max(q, 1) and the caustic map with probability q / max(q, 1), by Russian
     * roulette (photon_mapper.cpp:733-745, 1455-1462); a stored photon keeps its power, and the maps
     * are scaled by the inverse probabilities when they are built */
    float caustics_quality;
} liar_photon_desc;
typedef struct liar_photon_buffers {  /* device arrays of `capacity` photons */
    float* position;   /* x 3 */
    float* omega_in;   /* x 3: direction toward where the photon came from */
    float* power;      /* x 3: XYZ */
    uint32_t* path;    /* index of the emitted photon */
    uint32_t* tag;     /* map kinds (bits 0-1: LIAR_PHOTON_GLOBAL | LIAR_PHOTON_CAUSTIC) | bounce << 8 */
    uint64_t capacity;
    float* normal;     /* x 3, may be NULL: the shading normal on the side the photon came from */
} liar_photon_buffers;
typedef struct liar_photon_counts {
    uint64_t stored, global, caustic, emitted;
} liar_photon_counts;
int liar_gpu_photon_trace(liar_gpu_ctx* ctx, const liar_gpu_scene* scene, const liar_photon_desc* desc,
                          const liar_photon_buffers* out, liar_photon_counts* counts, void* stream);
/* The photon maps of the last PhotonMapper render on ctx (kept for the next render of the same
 * scene and settings): [0] photons shot, [1] global map size, [2] caustic map size, [3] 1 when maps
 * exist; radii (2 floats, may be NULL): the global and caustic estimation radii in use.
 * (PhotonMapper::doPreProcess statistics, src/liar/tracers/photon_mapper.cpp:372-390.) */
int liar_gpu_photon_mapper_stats(const liar_gpu_ctx* ctx, unsigned long long* out4, float* radii);
/* Copies map `map` (0 global, 1 caustic) of those maps to host arrays of `capacity` photons (any may
 * be NULL): positions, directions toward where the photons came from and scaled XYZ powers (n x 3
 * floats each), and the powers' recovery blends (n x 3 indices, n x 3 weights); *n_out = photons. */
int liar_gpu_photon_mapper_get_map(liar_gpu_ctx* ctx, int map, float* position, float* omega_in, float* power,
                                   int32_t* blend_idx, float* blend_w, size_t capacity, size_t* n_out);
/* Copies the irradiance map of those maps (final gathering, buildIrradianceMap,
 * src/liar/tracers/photon_mapper.cpp:970-995): positions, normals, irradiances (XYZ), their recovery
 * blends (n x 3 each) and squared estimation radii (n); any may be NULL; *n_out = points. */
int liar_gpu_photon_mapper_get_irradiance(liar_gpu_ctx* ctx, float* position, float* normal, float* xyz,
                                          int32_t* blend_idx, float* blend_w, float* r2, size_t capacity,
                                          size_t* n_out);

/* Allocation-free closest hit / any hit. It has no counterpart in the reference; it exists for
 * callers that must not call cudaMalloc while they trace: an application whose own pool
 * allocator owns the device memory, a frame loop whose other streams would be stalled by the
 * synchronisation cudaMalloc/cudaFree can cause, a plugin with a fixed memory budget.
 * Results are those of liar_gpu_trace_device (same kernel, same rules), without a context: the
 * work counter and status word live in a 256-byte device array compiled into the library.
 *   - d_rays / d_hits are the caller's device buffers on the mesh's device (16- / 8-byte
 *     aligned); at most 2^31 rays per call, more returns LIAR_ERR_INVALID.
 *   - The call allocates nothing. It reads the kernel's status word back on `stream` (NULL =
 *     the legacy default stream) and waits for that stream alone, so that it can return the
 *     status (LIAR_ERR_STACK on a traversal stack overflow); other streams are not waited for.
 *   - The first call on a device does the set-up: it looks up the array's device address
 *     (cudaGetSymbolAddress) with that device current and sizes the kernel's grid from its
 *     occupancy; later calls make no such queries. Make that first call before any stream
 *     capture. The kernel is the one the context path runs with its default launch shape, so
 *     once the program has traced through a context, the CUDA driver has its code loaded.
 *   - Every call shares the one array per device: calls that overlap on the GPU (from several
 *     host threads or streams at once) race on it and must be serialised by the caller. */
int liar_gpu_trace_device_noalloc(const liar_gpu_mesh* mesh, const liar_ray* d_rays, size_t n_rays,
                                  liar_hit* d_hits, int any_hit, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LIAR_GPU_H */
