"""Analytic spheres (scenery/sphere.cpp): their flattening, the exact ray/sphere test of the
oracle against double precision, and the oracle's renders of an analytic sphere against a finely
tessellated one."""
import numpy as np
import pytest

import oracle
from liar_b200 import cameras, render as R, scenery, shaders, spectra, textures as tx, tracers


def test_flattening_keeps_spheres_analytic_where_it_can():
    a = scenery.Sphere((1, 2, 3), 0.5)
    a.shader = shaders.Lambert(tx.Constant(0.5))
    b = scenery.Sphere((0, 0, 0), 1.0)
    moved = scenery.Transformation(b, [[0, -2, 0, 1], [2, 0, 0, 0], [0, 0, 2, 5], [0, 0, 0, 1]])  # rotate, scale 2
    squashed = scenery.Transformation(scenery.Sphere((0, 0, 0), 1.0), [[1, 0, 0, 0], [0, 2, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1]])
    mesh = scenery.Sphere((5, 0, 0), 1.0, subdivisions=2)
    lamp = scenery.LightArea(scenery.Sphere((0, 5, 0), 0.2))
    flat = R.flatten(scenery.List([a, moved, squashed, mesh, lamp]))
    np.testing.assert_allclose(flat.spheres, [[1, 2, 3, 0.5], [1, 0, 5, 2.0]], rtol=1e-6)
    assert list(flat.sphere_object) == [0, 1]
    # the non-similar transformation, the explicit mesh and the light's surface are triangles
    assert flat.triangles.shape[0] == 20 * 4 ** 5 + 20 * 4 ** 2 + 20 * 4 ** 5
    assert flat.scene_radius > 0
    only = R.flatten(a)
    assert only.triangles.shape[0] == 0 and only.desc().n_spheres == 1


def test_oracle_sphere_test_against_double_precision():
    import ctypes as C
    lib = oracle.lib()
    f = lib.oracle_sphere_intersect
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_void_p]
    rng = np.random.default_rng(1)
    hits = 0
    for _ in range(2000):
        o = rng.uniform(-4, 4, 3).astype(np.float32)
        c = rng.uniform(-1, 1, 3).astype(np.float32)
        r = np.float32(rng.uniform(0.2, 2))
        d = rng.normal(size=3).astype(np.float32)
        t0, t1 = np.zeros(1, np.float32), np.zeros(1, np.float32)
        got = f(o.ctypes.data, d.ctypes.data, c.ctypes.data, r, t0.ctypes.data, t1.ctypes.data)
        od, dd, cd = o.astype(np.float64), d.astype(np.float64), c.astype(np.float64)
        a, b, cc = dd @ dd, (od - cd) @ dd, (od - cd) @ (od - cd) - float(r) ** 2
        disc = b * b - a * cc
        if disc < -1e-5 * (b * b + abs(a * cc)):
            assert not got
            continue
        if disc <= 1e-5 * (b * b + abs(a * cc)):
            continue   # grazing: either answer
        assert got
        hits += 1
        e0, e1 = (-b - np.sqrt(disc)) / a, (-b + np.sqrt(disc)) / a
        scale = np.sqrt(od @ od) + np.sqrt(cd @ cd) + float(r)
        assert abs(t0[0] - e0) * np.sqrt(a) <= 1e-5 * scale and abs(t1[0] - e1) * np.sqrt(a) <= 1e-5 * scale
    assert hits > 100


def _ball_scene(sphere):
    floor = scenery.Parallelogram((-3, -3, 0), (6, 0, 0), (0, 6, 0))
    floor.shader = shaders.Lambert(tx.Constant(0.5))
    sky = scenery.LightSky(tx.Constant(1.0))
    cam = cameras.PerspectiveCamera()
    cam.sky = (0, 0, 1)
    cam.position = (0, -4, 1.5)
    cam.lookAt((0, 0, 0.8))
    return scenery.List([floor, sphere, sky]), cam


@pytest.mark.parametrize("shader", ["lambert", "mirror", "checker"])
def test_oracle_analytic_sphere_matches_a_fine_mesh(shader):
    def make(sub):
        s = scenery.Sphere((0, 0, 0.8), 0.8, subdivisions=sub)
        if shader == "lambert":
            s.shader = shaders.Lambert(tx.Constant(0.7))
        elif shader == "mirror":
            s.shader = shaders.Mirror(tx.Constant(0.9))
        else:
            board = tx.CheckerBoard(tx.Constant(0.8), tx.Constant(0.1))
            board.antiAliasing = "none"
            s.shader = shaders.Lambert(tx.TransformationUv(board, [[8, 0, 0], [0, 4, 0], [0, 0, 1]]))
        return s
    t = tracers.AdjointPhotonTracer()
    t.maxRayGeneration = 3
    out = []
    for sub in (None, 6):
        scene, cam = _ball_scene(make(sub))
        img, _ = R.resolve(oracle.RenderScene(R.flatten(scene)).render(R.render_desc(cam, 48, 36, 32, t, seed=2)))
        out.append(img)
    a, b = out
    # the same picture up to the tessellation's silhouette pixels and the estimates' noise
    assert abs(a[..., 1].mean() / b[..., 1].mean() - 1) < 0.02
    assert np.mean(np.abs(a[..., 3] - b[..., 3]) > 0.05) < 0.03
