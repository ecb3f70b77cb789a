"""Ray tracers of the scene API (``liar.tracers``). AdjointPhotonTracer runs as the wavefront path
tracer of liar_b200/csrc/render.cu (src/liar/tracers/adjoint_photon_tracer.cpp)."""
from __future__ import annotations


class RayTracer:
    def __init__(self):
        self.maxRayGeneration = 8  # kernel/ray_tracer.cpp:171
        self.maxDepth = 0          # hard cap on generations (0 = none), see DESIGN.md


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
