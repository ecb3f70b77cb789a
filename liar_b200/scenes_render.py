"""Seeded synthetic render scenes built through the scene API (the workloads' stand-ins).

* :func:`cornell_box` -- the plain spectral path-tracing workload: a Cornell-style box of
  axis-aligned quads (5 Lambert walls: white 0.75; red and green as 3-knot piecewise-linear
  reflectances over 380-720 nm with knots at 380/550/720 nm: red (0.05, 0.12, 0.63), green
  (0.12, 0.63, 0.05)), the two rotated blocks of the classic Cornell box (12 triangles each,
  footprints from the reference's src/liar/tools/cornell_box.py), and a 0.25 x 0.25 ceiling
  area light with 2856 K blackbody emission; pinhole camera as in that tool.
* :func:`white_furnace` -- a Lambert(1) sphere under a constant LightSky(1), after the reference's
  test/white_furnace script: every pixel that sees the sphere must converge to Y = 1.
"""
from __future__ import annotations

import math

from . import cameras, samplers, scenery, shaders, spectra, textures, tracers

NM = 1e-9


def _s(*xyz):
    return tuple(0.01 * x for x in xyz)


def _block(footprint, heights):
    import numpy as np
    verts = [_s(p[0], h, p[1]) for h in heights for p in footprint]
    tri = [(0, 2, 1), (0, 3, 2), (4, 6, 7), (4, 5, 6), (0, 5, 4), (0, 1, 5),
           (1, 6, 5), (1, 2, 6), (2, 7, 6), (2, 3, 7), (3, 4, 7), (3, 0, 4)]
    return scenery.TriangleMesh(np.asarray(verts), [], [], np.asarray(tri))


def cornell_box(light_scale: float = 2000.0):
    """Returns (scene, camera) of the Cornell workload."""
    white = shaders.Lambert(textures.Constant(0.75))
    red = shaders.Lambert(textures.Constant(spectra.Sampled([380 * NM, 550 * NM, 720 * NM], [0.05, 0.12, 0.63])))
    green = shaders.Lambert(textures.Constant(spectra.Sampled([380 * NM, 550 * NM, 720 * NM], [0.12, 0.63, 0.05])))
    floor = scenery.Parallelogram(_s(0, 0, 559.2), _s(552.8, 0, 0), _s(0, 0, -559.2))
    ceiling = scenery.Parallelogram(_s(0.0, 548.8, 0), _s(556.0, 0, 0), _s(0, 0, 559.2))
    back = scenery.Parallelogram(_s(556, 0, 559.2), _s(-556.0, 0, 0), _s(0, 548.8, 0))
    right = scenery.Parallelogram(_s(0, 0, 559.2), _s(0, 0, -559.2), _s(0, 548.8, 0))
    left = scenery.Parallelogram(_s(552.8, 0, 0), _s(0, 0, 559.2), _s(0, 548.8, 0))
    for w in (floor, ceiling, back):
        w.shader = white
    right.shader = green
    left.shader = red
    short = _block([(130.0, 65.0), (82.0, 225.0), (240.0, 272.0), (290.0, 114.0)], [0.05, 165.0])
    tall = _block([(423.0, 247.0), (265.0, 296.0), (314.0, 456.0), (472.0, 406.0)], [0.05, 330.0])
    short.shader = white
    tall.shader = white
    radiance = spectra.BlackBody(2856.0, light_scale)
    surf = scenery.Parallelogram((2.78 - 0.125, 5.4879, 2.795 - 0.125), (0.25, 0.0, 0.0), (0.0, 0.0, 0.25))
    light = scenery.LightArea(surf)
    light.radiance = radiance
    light.numberOfEmissionSamples = 16
    light.shader = shaders.Sum([shaders.Unshaded(textures.Constant(radiance)), shaders.Lambert(textures.Constant(0.78))])
    scene = scenery.List([light, floor, ceiling, back, right, left, short, tall])
    cam = cameras.PerspectiveCamera()
    cam.aspectRatio = 1
    cam.fovAngle = 2 * math.atan((0.025 / 0.035) / 2)
    cam.position = _s(278, 273, -800)
    cam.sky = (0, 1, 0)
    cam.direction = (0, 0, 1)
    return scene, cam


def cornell_engine(width: int = 256, height: int = 256, spp: int = 16, max_ray_generation: int = 3,
                   max_depth: int = 8, seed: int = 0):
    """RenderEngine of the Cornell workload: 256 x 256, 16 spp, RR from generation 3, depth 8."""
    from .kernel import RenderEngine
    scene, cam = cornell_box()
    e = RenderEngine()
    e.scene = scene
    e.camera = cam
    e.sampler = samplers.Stratifier((width, height), spp)
    e.tracer = tracers.AdjointPhotonTracer()
    e.tracer.maxRayGeneration = max_ray_generation
    e.tracer.maxDepth = max_depth
    e.seed = seed
    return e


def white_furnace():
    """(scene, camera): Lambert(1) unit sphere (flattened, exact normals) under LightSky(1)."""
    ball = scenery.Sphere((0, 0, 0), 1.0, subdivisions=4)
    ball.shader = shaders.Lambert(textures.Constant(1.0))
    sky = scenery.LightSky(textures.Constant(1.0))
    scene = scenery.List([ball, sky])
    cam = cameras.PerspectiveCamera()
    cam.position = (0, -4, 0)
    cam.lookAt((0, 0, 0))
    cam.aspectRatio = 1
    cam.fovAngle = math.radians(30)
    return scene, cam


def photon_scene(light_scale: float = 50.0):
    """The photon-mapping workload: a glass sphere (Dielectric, Cauchy A = 1.5, B = 0.0042 um^2)
    and a tilted GGX copper panel (CookTorrance with copper n, k) under a 5000 K point light. The
    reference stores photons only on surfaces with a diffuse BSDF (photon_mapper.cpp:733), so the
    two objects stand on a Lambert ground plane that receives the caustics."""
    from . import scenery as sc
    ground = sc.Parallelogram((-3, 0, -3), (6, 0, 0), (0, 0, 6))
    ground.shader = shaders.Lambert(textures.Constant(0.7))
    ball = sc.Sphere((-0.4, 0.5, 0.2), 0.5, subdivisions=5)
    ball.shader = shaders.Dielectric(textures.Constant(spectra.Cauchy(1.5, 0.0042)))
    panel = sc.Parallelogram((0.6, 0.0, -0.8), (0.5, 0.0, 0.9), (0.3, 1.2, 0.0))
    cu = shaders.CookTorrance(textures.Constant(spectra.spd("Cu", "n")), textures.Constant(spectra.spd("Cu", "k")))
    cu.mdf = shaders.MicrofacetTrowbridgeReitz()
    cu.roughness = textures.Constant(0.15)
    panel.shader = cu
    light = sc.LightPoint((-0.2, 2.6, -0.6), spectra.BlackBody(5000.0, light_scale))
    scene = sc.List([ground, ball, panel, light])
    cam = cameras.PerspectiveCamera()
    cam.position = (0.0, 2.2, -3.6)
    cam.lookAt((0.0, 0.3, 0.0))
    cam.aspectRatio = 16 / 9
    return scene, cam
