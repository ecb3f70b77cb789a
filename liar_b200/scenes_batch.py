"""Seeded synthetic scenes for batched rendering: many procedural scenes of uneven size.

Each scene is a ground plane (a displaced grid) with a handful of displaced spheres (cube-spheres
with a sum-of-sines radial bump field) on it, lit by a constant sky and a 6500 K area light. Sphere
materials are drawn from Lambert, a GGX conductor (CookTorrance with the copper, gold or silver
n/k tables) of roughness U(0.05, 0.6), and a dielectric of index 1.5. Triangle count, square image
side and samples per pixel are each log-uniform in their ranges.

No reference counterpart (the reference renders one hand-built scene per script); scenes are built
through the same scene API (scenery / shaders / textures) as every other workload.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import cameras, scenery, shaders, spectra, textures, tracers


def cube_sphere(n: int, center, radius: float, rng: np.random.Generator, amplitude: float = 0.08):
    """A cube with every face cut into n x n quads, projected onto the sphere and displaced by
    r(d) = radius * (1 + amplitude * sum of 4 random sines of d). 12 n^2 triangles, outward winding."""
    g = np.linspace(-1.0, 1.0, n + 1)
    a, b = np.meshgrid(g, g, indexing="ij")
    a, b = a.ravel(), b.ravel()
    one = np.ones_like(a)
    faces = []
    # (axis permutation, sign) of the six faces; (u, v, w) -> xyz with w = +-1
    for axis in range(3):
        for sign in (1.0, -1.0):
            p = np.empty((a.size, 3))
            u_ax, v_ax = [k for k in range(3) if k != axis]
            p[:, axis] = sign * one
            p[:, u_ax] = a
            p[:, v_ax] = b * sign
            faces.append(p)
    pts = np.concatenate(faces)
    d = pts / np.linalg.norm(pts, axis=1, keepdims=True)
    bump = np.zeros(d.shape[0])
    for _ in range(4):
        w = rng.normal(size=3)
        w *= rng.uniform(2.0, 7.0) / np.linalg.norm(w)
        bump += np.sin(d @ w + rng.uniform(0, 2 * math.pi))
    r = radius * (1.0 + amplitude * bump / 4.0)
    verts = (d * r[:, None] + np.asarray(center, dtype=np.float64)).astype(np.float32)
    i = np.arange(n)
    q00 = (i[:, None] * (n + 1) + i[None, :]).ravel()
    q10, q01, q11 = q00 + (n + 1), q00 + 1, q00 + (n + 2)
    per_face = (n + 1) * (n + 1)
    tris = []
    for f in range(6):
        o = f * per_face
        t = np.concatenate([np.stack([q00, q10, q11], 1), np.stack([q00, q11, q01], 1)]) + o
        # orient outward: compare the winding normal with the position
        v0, v1, v2 = verts[t[:, 0]], verts[t[:, 1]], verts[t[:, 2]]
        nrm = np.cross(v1 - v0, v2 - v0)
        flip = np.einsum("ij,ij->i", nrm, v0 - np.asarray(center, dtype=np.float32)) < 0
        t[flip] = t[flip][:, [0, 2, 1]]
        tris.append(t)
    return verts, np.concatenate(tris).astype(np.uint32)


def ground_grid(nx: int, ny: int, half: float, rng: np.random.Generator, amplitude: float = 0.03):
    """A 2 nx ny-triangle grid over [-half, half]^2 at y ~ 0, gently displaced, facing +y."""
    x = np.linspace(-half, half, nx + 1)
    z = np.linspace(-half, half, ny + 1)
    X, Z = np.meshgrid(x, z, indexing="ij")
    Y = np.zeros_like(X)
    for _ in range(3):
        k = rng.normal(size=2)
        k *= rng.uniform(0.5, 2.0) / np.linalg.norm(k)
        Y += np.sin(k[0] * X + k[1] * Z + rng.uniform(0, 2 * math.pi))
    Y *= amplitude / 3.0
    verts = np.stack([X, Y, Z], -1).reshape(-1, 3).astype(np.float32)
    i, j = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    a = (i * (ny + 1) + j).ravel()
    b, c, d = a + (ny + 1), a + 1, a + (ny + 2)
    # +y facing: (a, c, d) and (a, d, b) wind counter-clockwise seen from above
    tris = np.concatenate([np.stack([a, c, d], 1), np.stack([a, d, b], 1)]).astype(np.uint32)
    return verts, tris


METALS = ("Cu", "Au", "Ag")


def _material(kind: str, rng: np.random.Generator):
    if kind == "lambert":
        return shaders.Lambert(textures.Constant(float(rng.uniform(0.2, 0.85))))
    if kind == "conductor":
        metal = METALS[int(rng.integers(len(METALS)))]
        m = shaders.CookTorrance(textures.Constant(spectra.spd(metal, "n")), textures.Constant(spectra.spd(metal, "k")))
        m.mdf = shaders.MicrofacetTrowbridgeReitz()
        m.roughness = textures.Constant(float(rng.uniform(0.05, 0.6)))
        return m
    return shaders.Dielectric(textures.Constant(1.5))


@dataclass
class BatchScene:
    scene: object
    camera: object
    width: int
    height: int
    spp: int
    n_triangles: int
    materials: tuple


def batch_scene(seed: int, n_triangles: int, side: int, spp: int) -> BatchScene:
    """One procedural scene of about n_triangles triangles (within a few percent)."""
    rng = np.random.default_rng(seed)
    n_spheres = int(rng.integers(3, 9))
    sphere_share = rng.uniform(0.4, 0.8)
    per_sphere = sphere_share * n_triangles / n_spheres
    objs, kinds = [], []
    used = 0
    placed = []
    for s in range(n_spheres):
        n = max(2, int(round(math.sqrt(per_sphere / 12.0))))
        radius = float(rng.uniform(0.25, 0.7))
        for _ in range(50):
            cx, cz = rng.uniform(-2.5, 2.5, size=2)
            if all((cx - px) ** 2 + (cz - pz) ** 2 > (radius + pr) ** 2 for px, pz, pr in placed):
                break
        placed.append((cx, cz, radius))
        v, t = cube_sphere(n, (cx, radius * 1.05, cz), radius, rng)
        mesh = scenery.TriangleMesh(v, [], [], t)
        kind = ("lambert", "conductor", "dielectric")[int(rng.integers(3))]
        mesh.shader = _material(kind, rng)
        objs.append(mesh)
        kinds.append(kind)
        used += t.shape[0]
    rest = max(n_triangles - used, 200)
    nx = max(10, int(round(math.sqrt(rest / 2.0))))
    ny = max(10, int(round(rest / (2.0 * nx))))
    gv, gt = ground_grid(nx, ny, 4.0, rng)
    ground = scenery.TriangleMesh(gv, [], [], gt)
    ground.shader = shaders.Lambert(textures.Constant(0.5))
    objs.append(ground)
    used += gt.shape[0]
    sky = scenery.LightSky(textures.Constant(0.3))
    panel = scenery.Parallelogram((-0.75, 4.0, -0.75), (0.0, 0.0, 1.5), (1.5, 0.0, 0.0))
    lamp = scenery.LightArea(panel)
    lamp.radiance = spectra.BlackBody(6500.0, float(rng.uniform(10.0, 20.0)))
    lamp.shader = shaders.Unshaded(textures.Constant(lamp.radiance))
    scene = scenery.List(objs + [sky, lamp])
    cam = cameras.PerspectiveCamera()
    ang = rng.uniform(0, 2 * math.pi)
    cam.position = (6.0 * math.cos(ang), float(rng.uniform(1.5, 3.0)), 6.0 * math.sin(ang))
    cam.sky = (0, 1, 0)
    cam.lookAt((0.0, 0.4, 0.0))
    cam.aspectRatio = 1.0
    cam.fovAngle = math.radians(50)
    return BatchScene(scene, cam, side, side, spp, used, tuple(kinds))


def _log_uniform_int(rng, lo: float, hi: float, size: int) -> np.ndarray:
    return np.round(np.exp(rng.uniform(math.log(lo), math.log(hi), size=size))).astype(np.int64)


def batch_workload_params(n_scenes: int = 64, seed: int = 0, tris=(10_000, 2_000_000), side=(128, 1024),
                          spp=(4, 64)) -> list[tuple[int, int, int, int]]:
    """(scene seed, triangle count, image side, samples per pixel) of each scene of the workload:
    triangle count, square image side and samples per pixel log-uniform in their ranges."""
    rng = np.random.default_rng(seed)
    nt = _log_uniform_int(rng, *tris, n_scenes)
    sd = _log_uniform_int(rng, *side, n_scenes)
    sp = _log_uniform_int(rng, *spp, n_scenes)
    seeds = rng.integers(0, 2**31, size=n_scenes)
    return [(int(seeds[k]), int(nt[k]), int(sd[k]), int(sp[k])) for k in range(n_scenes)]


def batch_workload(n_scenes: int = 64, seed: int = 0, tris=(10_000, 2_000_000), side=(128, 1024), spp=(4, 64)):
    """The batched-rendering workload: n_scenes scenes of batch_workload_params (all seeded)."""
    return [batch_scene(*p) for p in batch_workload_params(n_scenes, seed, tris, side, spp)]


def batch_tracer(max_ray_generation: int = 3, max_depth: int = 8):
    t = tracers.AdjointPhotonTracer()
    t.maxRayGeneration = max_ray_generation
    t.maxDepth = max_depth
    return t
