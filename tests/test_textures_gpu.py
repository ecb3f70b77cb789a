"""uv textures on the GPU (render_dev.cuh texture_eval / param_eval) against the oracle's
restatement (oracle_render.cpp texture / param) in every renderer that shades surfaces: the path
tracer, DirectLighting, the batched renderer and photon tracing; and the scene upload's checks of
texture trees."""
import numpy as np
import pytest
import torch

import oracle
from liar_b200 import batch as B, cameras, photons, render as R, scenery, shaders, spectra, textures as tx, tracers
from liar_b200._native import LiarGpuError
from liar_b200.kernel import default_context
from liar_b200.recovery import sRGB

pytestmark = pytest.mark.gpu


def _scene():
    a, b = tx.Constant(0.85), tx.Constant(spectra.Sampled([380e-9, 550e-9, 720e-9], [0.1, 0.3, 0.6]))
    board = tx.CheckerBoard(a, b)
    board.antiAliasing = "none"
    floor = scenery.Parallelogram((-2, 0, -2), (4, 0, 0), (0, 0, 4))
    floor.shader = shaders.Lambert(tx.TransformationUv(board, [[4, 0, 0.25], [0, 4, 0], [0, 0, 1]]))
    grid = tx.GridBoard(tx.Constant(0.05), tx.Constant(0.6))
    grid.thickness = (0.15, 0.3)
    back = scenery.Parallelogram((-2, 0, 2), (4, 0, 0), (0, 3, 0))
    back.shader = shaders.Lambert(tx.TransformationUv(grid, [[3, 1, 0], [0, 3, 0], [0, 0, 1]]))
    marble = scenery.Parallelogram((-1.9, 0, 1.9), (0, 0, -3), (0, 2.5, 0))    # the left wall
    marble.shader = shaders.Lambert(tx.Sum(0.3, tx.Product(0.6, tx.Abs(tx.FBm(4, 0.55)))))
    ball_noise = tx.Sum([0.5, tx.Product([0.45, tx.Perlin(9)])])
    ball = scenery.Sphere((-0.7, 0.6, 0.2), 0.6, subdivisions=3)
    ct = shaders.CookTorrance(tx.Constant(spectra.Spectrum(1.5)), tx.Constant(spectra.Spectrum(3.0)))
    stripes = tx.CheckerBoard(tx.Constant(1.0), tx.Constant(0.2))
    stripes.split = (0.5, 2.0)        # v always below the split: stripes along u
    stripes.antiAliasing = "none"
    ct.reflectance = tx.TransformationUv(stripes, [[8, 0, 0], [0, 1, 0], [0, 0, 1]])
    ct.roughness = tx.Constant(0.3)
    ct.absorptionCoefficient = ball_noise       # a noisy absorption: textures on non-reflectance slots too
    ball.shader = ct
    box = scenery.Box((0.3, 0, -0.5), (1.1, 0.8, 0.3))
    mirrored = scenery.Transformation(box, [[-1, 0, 0, 0.6], [0, 1, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1]])
    rng = np.random.default_rng(11)
    rgb = rng.uniform(0.05, 0.9, size=(5, 7, 3)).astype(np.float32)
    photo = tx.Image.from_xyz(sRGB.linearSpace().toXYZlinear(rgb), antiAliasing="bilinear")
    panel = scenery.Parallelogram((1.9, 0, -1.5), (0, 0, 3), (0, 2, 0))
    panel.shader = shaders.Lambert(tx.TransformationUv(photo, [[2, 0, 0.1], [0, 1.5, 0], [0, 0, 1]]))
    tiles = tx.Image.from_xyz(sRGB.linearSpace().toXYZlinear(rgb[:2, :3]), antiAliasing="none")
    box.shader = shaders.Lambert(tiles)
    surf = scenery.Parallelogram((-0.5, 2.5, -0.5), (1, 0, 0), (0, 0, 1))
    light = scenery.LightArea(surf)
    light.radiance = spectra.BlackBody(5000, 20)
    cam = cameras.PerspectiveCamera()
    cam.position = (0, 1.5, -4)
    cam.lookAt((0, 0.8, 0))
    return scenery.List([floor, back, marble, ball, mirrored, panel, light]), cam


def _within_3_sigma(g, c, min_fraction=0.99):
    mg, vg = R.resolve(g)
    mc, vc = R.resolve(c)
    sig = np.sqrt(vg + vc)
    ok = np.abs(mg[..., :3] - mc[..., :3]) <= 3 * sig + 1e-6 * np.maximum(np.abs(mc[..., :3]), 1.0)
    assert ok.mean() >= min_fraction, f"only {ok.mean():.4f} of pixel channels within 3 sigma"
    np.testing.assert_array_equal(g[..., 7], c[..., 7])
    assert abs(mg[..., 1].mean() / mc[..., 1].mean() - 1) < 0.02
    return mg, mc


@pytest.fixture(scope="module")
def textured():
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        scene, cam = _scene()
        flat = R.flatten(scene)
    assert flat.triangle_uvs is not None and len(flat.textures) >= 10 and flat.texture_pixels is not None
    return flat, R.GpuScene(default_context(), flat), cam


@pytest.mark.parametrize("kind", ["path", "direct"])
def test_textured_scene_matches_oracle(textured, kind):
    flat, gs, cam = textured
    if kind == "path":
        t = tracers.AdjointPhotonTracer()
    else:
        t = tracers.DirectLighting()
    t.maxRayGeneration = 3
    d = R.render_desc(cam, 48, 40, 16, t, seed=5)
    g = gs.render(d)
    c = oracle.RenderScene(flat).render(d)
    mg, _ = _within_3_sigma(g, c)
    # the board shows: the floor's pixels take both checker values
    assert np.ptp(mg[-8:, :, 1]) > 0.05


def test_textured_batch_matches_single_render(textured):
    _, gs, cam = textured
    t = tracers.AdjointPhotonTracer()
    t.maxRayGeneration = 3
    t.maxDepth = 8                      # the batched renderer's bounded path length
    d = R.render_desc(cam, 40, 32, 8, t, seed=2)
    film = torch.zeros((d.height, d.width, 8), dtype=torch.float32, device="cuda:0")
    gs.render_device(d, film.data_ptr())
    br = B.BatchRenderer(default_context(), [(gs, d)], B.make_config(hero=1))
    br.launch()
    torch.cuda.synchronize()
    a, b = br.films[0].cpu().numpy(), film.cpu().numpy()
    scale = max(float(np.abs(b[..., :7]).max()), 1e-6)
    np.testing.assert_allclose(a[..., :7], b[..., :7], rtol=2e-5, atol=2e-6 * scale)
    br.close()


def test_textured_photon_trace_matches_oracle(textured):
    flat, gs, _ = textured
    d = photons.photon_desc(3000, max_emitted=400_000, wave=8192, ray_traced_direct=False, seed=6)
    g, gc = photons.trace_photons(gs, d, capacity=400_000)
    c, cc = oracle.photon_trace(oracle.RenderScene(flat), d, 400_000)
    g = {k: v.cpu().numpy() for k, v in g.items()}
    assert gc["emitted"] == cc["emitted"]
    gkey = (g["path"].astype(np.int64) << 8) | ((g["tag"] >> 8) & 0xFF)
    ckey = (c["path"].astype(np.int64) << 8) | ((c["tag"] >> 8) & 0xFF)
    common, gi, ci = np.intersect1d(gkey, ckey, return_indices=True)
    assert len(common) >= 0.98 * len(ckey)
    np.testing.assert_allclose(g["power"][gi], c["power"][ci], rtol=2e-3, atol=1e-3)


def _upload(flat):
    return R.GpuScene(default_context(), flat)


def test_upload_refuses_bad_texture_trees():
    p = scenery.Parallelogram((0, 0, 0), (1, 0, 0), (0, 1, 0))
    board = tx.CheckerBoard(0.1, 0.9)
    board.antiAliasing = "none"
    p.shader = shaders.Lambert(board)
    flat = R.flatten(p)
    _upload(flat)                                       # the tree as flattened is fine
    root = flat.materials[0].tex[0]
    flat.textures[flat.textures[root].a].type = R.TEX_UV_TRANSFORM
    flat.textures[flat.textures[root].a].a = root       # a cycle
    with pytest.raises(LiarGpuError):
        _upload(flat)
    flat = R.flatten(p)
    flat.materials[0].tex[0] = len(flat.textures)       # out of range
    with pytest.raises(LiarGpuError):
        _upload(flat)
    img = tx.Image.from_xyz(np.full((2, 2, 3), 0.5, np.float32))
    p.shader = shaders.Lambert(img)
    flat = R.flatten(p)
    _upload(flat)
    flat.textures[flat.materials[0].tex[0]].pixels = 2     # runs past the pool's end
    with pytest.raises(LiarGpuError):
        _upload(flat)
    deep = tx.Constant(0.5)
    for _ in range(40):
        deep = tx.TransformationUv(deep, [[1, 0, 0.01], [0, 1, 0], [0, 0, 1]])
    p.shader = shaders.Lambert(deep)
    with pytest.raises(LiarGpuError):
        _upload(R.flatten(p))


def _filtered_scene():
    """The reference's default filtering: CheckerBoard with bilinear anti-aliasing, Image with
    trilinear lookups over anisotropic (and, on a second panel, isotropic) mip levels, FBm whose
    octaves follow the footprint; a receding floor so that footprints grow across the image, and
    a thin-lens camera, whose differential rays start at the lens sample."""
    fine = tx.CheckerBoard(tx.Constant(0.9), tx.Constant(0.1))     # antiAliasing: the default, bilinear
    floor = scenery.Parallelogram((-3, 0, -2), (6, 0, 0), (0, 0, 30))
    floor.shader = shaders.Lambert(tx.TransformationUv(fine, [[12, 0, 0], [0, 60, 0], [0, 0, 1]]))
    rng = np.random.default_rng(3)
    pix = rng.uniform(0.05, 0.9, size=(37, 53, 3)).astype(np.float32)   # odd sizes: odd mip reductions
    aniso = tx.Image.from_xyz(sRGB.linearSpace().toXYZlinear(pix), antiAliasing="trilinear", mipMapping="anisotropic")
    back = scenery.Parallelogram((-3, 0, 6), (6, 0, 0), (0, 3, 0))
    back.shader = shaders.Lambert(tx.TransformationUv(aniso, [[6, 0, 0], [0, 2, 0], [0, 0, 1]]))
    iso = tx.Image.from_xyz(sRGB.linearSpace().toXYZlinear(pix[:16, :16]), antiAliasing="trilinear",
                            mipMapping="isotropic")
    side = scenery.Parallelogram((2.9, 0, -1), (0, 0, 8), (0, 2.5, 0))
    side.shader = shaders.Lambert(tx.TransformationUv(iso, [[5, 0, 0], [0, 3, 0], [0, 0, 1]]))
    ball = scenery.Sphere((-1.0, 0.7, 1.5), 0.7)
    ball.shader = shaders.Lambert(tx.Sum(0.25, tx.Product(0.5, tx.Abs(tx.FBm(8, 0.6)))))
    sky = scenery.LightSky(tx.Constant(0.7))
    lamp = scenery.LightArea(scenery.Parallelogram((-0.5, 3.5, 0.5), (1, 0, 0), (0, 0, 1)))
    lamp.radiance = spectra.BlackBody(5000, 10)
    cam = cameras.PerspectiveCamera()
    cam.position = (0, 1.2, -2.5)
    cam.lookAt((0, 0.6, 2.0))
    cam.lensRadius = 0.02
    cam.focusDistance = 4.0
    return scenery.List([floor, back, side, ball, sky, lamp]), cam


@pytest.mark.parametrize("kind", ["path", "direct"])
def test_filtered_textures_match_oracle(kind):
    scene, cam = _filtered_scene()
    flat = R.flatten(scene)
    assert flat.textures[flat.materials[0].tex[0]].type == R.TEX_UV_TRANSFORM
    gs = R.GpuScene(default_context(), flat)
    t = tracers.AdjointPhotonTracer() if kind == "path" else tracers.DirectLighting()
    t.maxRayGeneration = 3
    d = R.render_desc(cam, 64, 48, 9, t, seed=8)
    g = gs.render(d)
    c = oracle.RenderScene(flat).render(d)
    mg, _ = _within_3_sigma(g, c)
    # far down the floor the checkers are averaged: the top rows of the floor are near grey
    assert mg[..., 1].mean() > 0.05
    gs.close()


def test_filtered_textures_batch_matches_single_render():
    scene, cam = _filtered_scene()
    gs = R.GpuScene(default_context(), R.flatten(scene))
    t = tracers.AdjointPhotonTracer()
    t.maxRayGeneration = 3
    t.maxDepth = 8
    d = R.render_desc(cam, 40, 30, 4, t, seed=2)
    film = torch.zeros((d.height, d.width, 8), dtype=torch.float32, device="cuda:0")
    gs.render_device(d, film.data_ptr())
    br = B.BatchRenderer(default_context(), [(gs, d)], B.make_config(hero=1))
    br.launch()
    torch.cuda.synchronize()
    a, b = br.films[0].cpu().numpy(), film.cpu().numpy()
    scale = max(float(np.abs(b[..., :7]).max()), 1e-6)
    np.testing.assert_allclose(a[..., :7], b[..., :7], rtol=2e-5, atol=2e-6 * scale)
    br.close()
    gs.close()
