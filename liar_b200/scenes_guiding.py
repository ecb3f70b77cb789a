"""The learned-guiding workload: a closed room lit through a slit (seeded, synthetic).

A 10 x 10 x 4 room (x, z in [-5, 5], y in [0, 4]) of Lambert 0.75 walls and ceiling; the floor is
a GGX conductor (CookTorrance, MicrofacetTrowbridgeReitz, aluminium n/k, alpha = 0.2, i.e. linear
roughness sqrt(0.2)); the wall at x = +5 has one vertical 0.2 x 2 slit (z in [-0.1, 0.1],
y in [1, 3]) through which a 6500 K area light outside the room shines in; the room holds a seeded
clutter of random boxes (12 triangles each, about 200k triangles by default) standing on the floor
or floating below 2 m. The camera looks across the room from the corner opposite the slit.
No reference counterpart (the reference ships no such scene); built through the scene API.
"""
from __future__ import annotations

import math

import numpy as np

from . import cameras, scenery, shaders, spectra, textures, tracers


def _boxes(n: int, rng: np.random.Generator):
    """n boxes as one triangle mesh: sizes U(0.05, 0.25), rotated about y, 70% on the floor, the
    rest floating below 2 m; kept out of a 1 m band inside the slit wall."""
    size = rng.uniform(0.05, 0.25, size=(n, 3))
    cx = rng.uniform(-4.7, 3.8, size=n)
    cz = rng.uniform(-4.7, 4.7, size=n)
    on_floor = rng.random(n) < 0.7
    cy = np.where(on_floor, size[:, 1] / 2, rng.uniform(0.3, 2.0, size=n))
    ang = rng.uniform(0, 2 * math.pi, size=n)
    corners = np.array([[x, y, z] for y in (-0.5, 0.5) for x in (-0.5, 0.5) for z in (-0.5, 0.5)])  # 8 x 3
    local = corners[None] * size[:, None, :]
    c, s = np.cos(ang)[:, None], np.sin(ang)[:, None]
    x = local[..., 0] * c - local[..., 2] * s
    z = local[..., 0] * s + local[..., 2] * c
    verts = np.stack([x + cx[:, None], local[..., 1] + cy[:, None], z + cz[:, None]], -1).reshape(-1, 3)
    # corner index = 4 * (y > 0) + 2 * (x > 0) + (z > 0); faces wound outward
    quads = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    tri = []
    for a, b, cc, d in quads:
        tri += [(a, b, cc), (a, cc, d)]
    tri = np.asarray(tri)
    tris = (tri[None] + 8 * np.arange(n)[:, None, None]).reshape(-1, 3)
    return verts.astype(np.float32), tris.astype(np.uint32)


def slit_room(n_triangles: int = 200_000, seed: int = 0, light_scale: float = 400.0):
    """Returns (scene, camera) of the guiding workload."""
    rng = np.random.default_rng(seed)
    white = shaders.Lambert(textures.Constant(0.75))
    P = scenery.Parallelogram
    walls = [
        P((-5, 4, -5), (10, 0, 0), (0, 0, 10)),            # ceiling, facing down
        P((-5, 0, -5), (0, 4, 0), (10, 0, 0)),             # z = -5
        P((-5, 0, 5), (10, 0, 0), (0, 4, 0)),              # z = +5
        P((-5, 0, -5), (0, 0, 10), (0, 4, 0)),             # x = -5
        # x = +5 around the slit (z in [-0.1, 0.1], y in [1, 3])
        P((5, 0, -5), (0, 4, 0), (0, 0, 4.9)),
        P((5, 0, 0.1), (0, 4, 0), (0, 0, 4.9)),
        P((5, 0, -0.1), (0, 1, 0), (0, 0, 0.2)),
        P((5, 3, -0.1), (0, 1, 0), (0, 0, 0.2)),
    ]
    for w in walls:
        w.shader = white
    floor = P((-5, 0, -5), (0, 0, 10), (10, 0, 0))
    al = shaders.CookTorrance(textures.Constant(spectra.spd("Al", "n")), textures.Constant(spectra.spd("Al", "k")))
    al.mdf = shaders.MicrofacetTrowbridgeReitz()
    al.roughness = textures.Constant(math.sqrt(0.2))
    floor.shader = al
    n_boxes = max(1, n_triangles // 12)
    bv, bt = _boxes(n_boxes, rng)
    clutter = scenery.TriangleMesh(bv, [], [], bt)
    clutter.shader = white
    # the light: a 3 x 3 panel 1 m outside the slit, facing the room (-x)
    panel = P((6, 0.5, -1.5), (0, 0, 3), (0, 3, 0))
    lamp = scenery.LightArea(panel)
    lamp.radiance = spectra.BlackBody(6500.0, light_scale)
    scene = scenery.List(walls + [floor, clutter, lamp])
    cam = cameras.PerspectiveCamera()
    cam.position = (-4.5, 1.7, -4.5)
    cam.sky = (0, 1, 0)
    cam.lookAt((2.0, 1.0, 2.5))
    cam.aspectRatio = 1.0
    cam.fovAngle = math.radians(75)
    return scene, cam


def guiding_tracer(max_ray_generation: int = 3, max_depth: int = 8):
    t = tracers.AdjointPhotonTracer()
    t.maxRayGeneration = max_ray_generation
    t.maxDepth = max_depth
    return t
