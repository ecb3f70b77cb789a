"""Ray tracers of the scene API (``liar.tracers``). AdjointPhotonTracer runs as the wavefront path
tracer of liar_b200/csrc/render.cu (src/liar/tracers/adjoint_photon_tracer.cpp), DirectLighting and
PhotonMapper as the task wavefront of liar_b200/csrc/direct.cu (src/liar/tracers/direct_lighting.cpp,
photon_mapper.cpp)."""
from __future__ import annotations


class RayTracer:
    def __init__(self):
        self.maxRayGeneration = 8  # kernel/ray_tracer.cpp:171
        # hard cap on generations (0 = none), an extension: with Russian roulette from generation
        # maxRayGeneration it bounds the path length, as a fixed-depth workload asks
        self.maxDepth = 0


class AdjointPhotonTracer(RayTracer):
    kind = 0


class DirectLighting(RayTracer):
    """Whitted-style direct lighting (src/liar/tracers/direct_lighting.cpp): direct light by light
    and BSDF sampling per light, recursive specular (and glossy) reflection and transmission."""
    kind = 1

    def __init__(self):
        super().__init__()
        self.numberOfSecondaryLightSamples = 1   # direct_lighting.cpp:46-49
        self.traceGlossy = True


class PhotonMapper(DirectLighting):
    """Photon mapping (src/liar/tracers/photon_mapper.cpp): DirectLighting plus, at every vertex with
    a diffuse part, the caustic map's Gaussian-filtered estimate and the global map's radiance
    estimate; the maps are filled from the lights before rendering. With numFinalGatherRays > 0
    (and isRayTracingDirect) high-quality diffuse vertices gather the indirect light with that many
    BSDF-sampled rays, evaluated at their hits from the precomputed irradiance map
    (ratioPrecomputedIrradiance of the global photons), with numSecondaryGatherRays more rays where a
    hit lies closer than the estimation radius. Defaults as the reference's
    (photon_mapper.cpp:108-142); causticsQuality sets the storage probabilities of the two maps
    (1 / max(q, 1) global, q / max(q, 1) caustic, :1455-1462). Volumetric maps are not on the GPU
    path (participating media are out of scope)."""
    kind = 2
    MAP_TYPES = {"global": 0, "caustic": 1, "caustics": 1}

    def __init__(self):
        super().__init__()
        self.maxNumberOfPhotons = 100_000_000
        self.globalMapSize = 10_000
        self.causticsQuality = 1.0
        self.numFinalGatherRays = 0
        self.numSecondaryGatherRays = 1
        self.ratioPrecomputedIrradiance = 0.25
        self.isVisualizingPhotonMap = False
        self.isRayTracingDirect = True
        self._radius = [0.0, 0.0]
        self._tolerance = [0.05, 0.05]
        self._size = [50, 50]

    def _map(self, mapType: str) -> int:
        try:
            return self.MAP_TYPES[mapType]
        except KeyError:
            raise KeyError(f"map type must be 'global' or 'caustic', not {mapType!r}") from None

    def estimationRadius(self, mapType: str) -> float:
        return self._radius[self._map(mapType)]

    def setEstimationRadius(self, mapType: str, radius: float) -> None:
        self._radius[self._map(mapType)] = float(radius)

    def estimationTolerance(self, mapType: str) -> float:
        return self._tolerance[self._map(mapType)]

    def setEstimationTolerance(self, mapType: str, tolerance: float) -> None:
        self._tolerance[self._map(mapType)] = float(tolerance)

    def estimationSize(self, mapType: str) -> int:
        return self._size[self._map(mapType)]

    def setEstimationSize(self, mapType: str, size: int) -> None:
        self._size[self._map(mapType)] = int(size)
