// photon_mapper.h -- the photon maps a PhotonMapper render reads (src/liar/tracers/photon_mapper.cpp),
// shared by the map builder (photon_mapper.cu) and the DirectLighting wavefront that shades with
// them (direct.cu).
#pragma once
#include <stdint.h>

#include "../../include/liar_gpu.h"
#include "recovery.cuh"

namespace liar_gpu {

enum PmMapKind { kPmGlobal = 0, kPmCaustic = 1 };

// PhotonMapper's storage probabilities (photon_mapper.cpp:1455-1462) of causticsQuality q (0: the
// reference's 1, negative: 0): the global map 1 / max(q, 1), the caustic map q / max(q, 1)
inline void storage_probabilities(float quality, float& p_global, float& p_caustic) {
    const float q = quality == 0.0f ? 1.0f : (quality > 0.0f ? quality : 0.0f);
    const float m = q > 1.0f ? q : 1.0f;
    p_global = 1.0f / m;
    p_caustic = q / m;
}

// one photon map on the device: the photons in the reference's buffer order (emission, then
// bounce), their power scaled by 1 / photons emitted, and each power's spectral blend
struct PmMap {
    const liar_gpu_photon_map* grid = nullptr;  // gather structure over the positions
    const float* position = nullptr;            // n x 3
    const float* omega_in = nullptr;            // n x 3, toward where the photon came from
    const float* power = nullptr;               // n x 3, XYZ
    const int32_t* blend_idx = nullptr;         // n x 3 (RecoveryBlend of the power)
    const float* blend_w = nullptr;             // n x 3
    uint64_t n = 0;
    float radius = 0.0f;                        // estimationRadius (rMax of the gathers)
    int k = 0;                                  // estimationSize (kMax of the gathers)
};

// the precomputed irradiance map of final gathering (buildIrradianceMap, photon_mapper.cpp:970-995):
// points at a random subset of the global photons, each with its normal, its irradiance
// (estimateIrradianceImpl over the global map) as a recovery blend, and its squared radius
struct PmIrradiance {
    const liar_gpu_photon_map* grid = nullptr;  // nearest-neighbour structure over the points
    const float* position = nullptr;            // n x 3
    const float* normal = nullptr;              // n x 3
    const float* xyz = nullptr;                 // n x 3
    const int32_t* blend_idx = nullptr;         // n x 3
    const float* blend_w = nullptr;             // n x 3
    const float* r2 = nullptr;                  // n: squaredEstimationRadius (0: no photon found)
    uint64_t n = 0;
};

struct PmMaps {
    PmMap map[2];
    PmIrradiance irr;
    DRecovery rec;
    int visualize = 0;     // isVisualizingPhotonMap
    int ray_direct = 1;    // isRayTracingDirect
    int fg_rays = 0;       // numFinalGatherRays when final gathering is on (hasFinalGather), else 0
    int fg_secondary = 0;  // numSecondaryGatherRays
    uint64_t emitted = 0;  // photons shot
};

namespace rt {
int render_direct(liar_gpu_ctx* ctx, const liar_gpu_scene* scene, const liar_render_desc& R, float* d_film,
                  cudaStream_t st, const PmMaps* pm);
}  // namespace rt

}  // namespace liar_gpu
