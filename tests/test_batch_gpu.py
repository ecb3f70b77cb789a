"""Batched rendering (one CUDA-graph launch over many scenes) against single-scene renders and,
for scenes of the batched workload itself, against the CPU restatement of the reference.

With one hero wavelength the batch draws exactly the samples liar_gpu_render_device draws for each
item on its own, so the films agree to float rounding (only the order of the per-pixel atomic adds
differs); the single-scene renderer itself is checked against the CPU restatement of the reference
in test_render_gpu.py. Four hero wavelengths change the estimator, not its expectation: images
agree with the one-wavelength images within 3 sigma.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle
from liar_b200 import (batch as B, cameras, render as R, scenery, scenes_batch, scenes_render, shaders, spectra,
                       textures, tracers)
from liar_b200._native import LiarGpuError
from liar_b200.kernel import default_context

pytestmark = pytest.mark.gpu


def _tracer(max_gen=3, max_depth=8):
    t = tracers.AdjointPhotonTracer()
    t.maxRayGeneration = max_gen
    t.maxDepth = max_depth
    return t


def _single(gs, desc):
    film = torch.zeros((desc.height, desc.width, 8), dtype=torch.float32, device="cuda:0")
    gs.render_device(desc, film.data_ptr())
    torch.cuda.synchronize()
    return film.cpu().numpy()


def _close(a, b):
    scale = max(float(np.abs(b[..., :7]).max()), 1e-6)
    np.testing.assert_allclose(a[..., :7], b[..., :7], rtol=2e-5, atol=2e-6 * scale)
    np.testing.assert_array_equal(a[..., 7], b[..., 7])


def _mean_within(a, b, sigmas=3.0, min_fraction=0.99):
    ma, va = R.resolve(a)
    mb, vb = R.resolve(b)
    sig = np.sqrt(va + vb)
    ok = np.abs(ma[..., :3] - mb[..., :3]) <= sigmas * sig + 1e-6 * np.maximum(np.abs(mb[..., :3]), 1.0)
    assert ok.mean() >= min_fraction, f"only {ok.mean():.4f} of pixel channels within {sigmas} sigma"
    return ma, mb


@pytest.fixture(scope="module")
def cornell():
    scene, cam = scenes_render.cornell_box()
    return R.GpuScene(default_context(), R.flatten(scene)), cam


def test_single_item_matches_single_render(cornell):
    gs, cam = cornell
    desc = R.render_desc(cam, 64, 64, 8, _tracer(), seed=3)
    ref = _single(gs, desc)
    br = B.BatchRenderer(default_context(), [(gs, desc)], B.make_config(hero=1))
    br.launch()
    torch.cuda.synchronize()
    _close(br.films[0].cpu().numpy(), ref)
    st = br.stats()
    assert st["paths"] == 64 * 64 * 8 and st["waves"] == 1
    assert st["segments"] >= st["paths"] and st["hits"] <= st["segments"]
    br.close()


def test_many_items_many_waves_match(cornell):
    """Items of different sizes, a second scene, repeated scenes and waves that straddle items."""
    ctx = default_context()
    gs, cam = cornell
    wf_scene, wf_cam = scenes_render.white_furnace()
    wf = R.GpuScene(ctx, R.flatten(wf_scene))
    entries = [
        (gs, R.render_desc(cam, 40, 24, 3, _tracer(), seed=1)),
        (wf, R.render_desc(wf_cam, 33, 17, 5, _tracer(2, 5), seed=2)),
        (gs, R.render_desc(cam, 16, 16, 1, _tracer(1, 3), seed=9, first_sample=7)),
        (wf, R.render_desc(wf_cam, 64, 64, 2, _tracer(), seed=4)),
    ]
    refs = [_single(g, d) for g, d in entries]
    br = B.BatchRenderer(ctx, entries, B.make_config(hero=1, wave_paths=1000))
    br.launch()
    torch.cuda.synchronize()
    for film, ref in zip(br.films, refs):
        _close(film.cpu().numpy(), ref)
    total = sum(d.width * d.height * d.spp for _, d in entries)
    st = br.stats()
    assert st["paths"] == total and st["waves"] == -(-total // 1000)
    # a second launch renders the same samples again: the films double
    first = [f.clone() for f in br.films]
    br.launch()
    torch.cuda.synchronize()
    for f, f0 in zip(br.films, first):
        torch.testing.assert_close(f, 2 * f0, rtol=1e-5, atol=1e-5 * float(f0.abs().max()))
    br.close()


def test_hero_wavelengths_same_expectation(cornell):
    gs, cam = cornell
    d = R.render_desc(cam, 32, 32, 64, _tracer(), seed=5)
    one = B.BatchRenderer(default_context(), [(gs, d)], B.make_config(hero=1))
    four = B.BatchRenderer(default_context(), [(gs, d)], B.make_config(hero=4))
    one.launch()
    four.launch()
    torch.cuda.synchronize()
    a, b = four.films[0].cpu().numpy(), one.films[0].cpu().numpy()
    ma, mb = _mean_within(a, b)
    # the luminance of the lit surfaces (the light, a sub-pixel emitter far brighter than the rest
    # and seen by the camera, would dominate the mean with its variance)
    lit = (ma[..., 1] < 2.0) & (mb[..., 1] < 2.0)
    assert abs(ma[..., 1][lit].mean() / mb[..., 1][lit].mean() - 1) < 0.02
    # hero wavelengths cut the colour noise: the mean per-pixel variance of X and Z drops
    _, va = R.resolve(a)
    _, vb = R.resolve(b)
    assert va[..., 0].mean() < vb[..., 0].mean() and va[..., 2].mean() < vb[..., 2].mean()


def test_white_furnace_hero():
    """Lambert(1) sphere under a unit sky: every pixel that sees the sphere converges to Y = 1."""
    scene, cam = scenes_render.white_furnace()
    gs = R.GpuScene(default_context(), R.flatten(scene))
    d = R.render_desc(cam, 32, 32, 64, _tracer(64, 64), seed=11)
    br = B.BatchRenderer(default_context(), [(gs, d)], B.make_config(hero=4))
    br.launch()
    torch.cuda.synchronize()
    m, v = R.resolve(br.films[0].cpu().numpy())
    # pixels whose whole footprint is well inside the unit sphere's silhouette
    cd = cam.flatten()
    ys, xs = np.mgrid[0:32, 0:32]
    sx, sy = (xs + 0.5) / 32 - 0.5, (ys + 0.5) / 32 - 0.5
    dirs = (np.asarray(cd["direction"])[None, None] + sx[..., None] * np.asarray(cd["right"])
            + sy[..., None] * np.asarray(cd["down"]))
    dirs /= np.linalg.norm(dirs, axis=-1, keepdims=True)
    o = np.asarray(cd["position"])
    inside = (dirs @ o) ** 2 - (o @ o - 1.0) > 0.25
    assert inside.sum() > 50
    y = m[..., 1][inside]
    sig = np.sqrt(v[..., 1][inside].mean() / inside.sum())
    assert abs(y.mean() - 1.0) < max(4 * sig, 5e-3)


def test_dispersive_glass_hero():
    """A Cauchy-dispersion glass sphere on a Lambert ground under an area light: past the glass the
    path carries one wavelength; the 4-wavelength image keeps the 1-wavelength expectation."""
    ground = scenery.Parallelogram((-3, 0, -3), (0, 0, 6), (6, 0, 0))
    ground.shader = shaders.Lambert(textures.Constant(0.7))
    ball = scenery.Sphere((0, 0.6, 0), 0.6, subdivisions=4)
    ball.shader = shaders.Dielectric(textures.Constant(spectra.Cauchy(1.5, 0.0042)))
    lamp = scenery.LightArea(scenery.Parallelogram((-0.5, 2.5, -0.5), (1, 0, 0), (0, 0, 1)))
    lamp.radiance = spectra.BlackBody(5000, 20)
    cam = cameras.PerspectiveCamera()
    cam.position = (0, 1.6, -3.5)
    cam.sky = (0, 1, 0)
    cam.lookAt((0, 0.4, 0))
    cam.aspectRatio = 16 / 9
    gs = R.GpuScene(default_context(), R.flatten(scenery.List([ground, ball, lamp])))
    d = R.render_desc(cam, 48, 27, 256, _tracer(3, 8), seed=13)
    one = B.BatchRenderer(default_context(), [(gs, d)], B.make_config(hero=1))
    four = B.BatchRenderer(default_context(), [(gs, d)], B.make_config(hero=4))
    one.launch()
    four.launch()
    torch.cuda.synchronize()
    ma, mb = _mean_within(four.films[0].cpu().numpy(), one.films[0].cpu().numpy(), min_fraction=0.985)
    assert mb[..., 1].mean() > 0.05
    assert abs(ma[..., 1].mean() / mb[..., 1].mean() - 1) < 0.03


def test_procedural_batch_matches_single_renders():
    """Scenes of the batched workload (spheres of three material kinds on a ground grid)."""
    ctx = default_context()
    scenes = [scenes_batch.batch_scene(s, n, 48, 4) for s, n in ((1, 20_000), (2, 60_000), (3, 12_000))]
    entries = []
    for bs in scenes:
        gs = R.GpuScene(ctx, R.flatten(bs.scene))
        entries.append((gs, R.render_desc(bs.camera, bs.width, bs.height, bs.spp, scenes_batch.batch_tracer(), seed=21)))
    refs = [_single(g, d) for g, d in entries]
    br = B.BatchRenderer(ctx, entries, B.make_config(hero=1, wave_paths=5000))
    br.launch()
    torch.cuda.synchronize()
    for film, ref in zip(br.films, refs):
        _close(film.cpu().numpy(), ref)
        assert film[..., 1].sum().item() > 0


def test_workload_scenes_through_the_batch_match_the_oracle():
    """The smallest, the median and the largest scene of the 64-scene workload (by triangles: 10k
    to 2M), rendered together in one 4-hero-wavelength graph launch at 40 x 40 x 16 spp, against
    the oracle's one-wavelength restatement of the reference's path tracer on the same scenes."""
    ctx = default_context()
    params = scenes_batch.batch_workload_params(64, seed=0)
    order = np.argsort([p[1] for p in params])
    picks = [int(order[0]), int(order[len(order) // 2]), int(order[-1])]
    assert params[picks[0]][1] < 12_000 and params[picks[-1]][1] > 1_500_000
    flats, entries = [], []
    for k in picks:
        bs = scenes_batch.batch_scene(params[k][0], params[k][1], 40, 16)
        flats.append(R.flatten(bs.scene))
        gs = R.GpuScene(ctx, flats[-1])
        entries.append((gs, R.render_desc(bs.camera, 40, 40, 16, scenes_batch.batch_tracer(), seed=100 + k)))
    br = B.BatchRenderer(ctx, entries, B.make_config(hero=4))
    br.launch()
    torch.cuda.synchronize()
    for film, flat, (gs, d) in zip(br.films, flats, entries):
        c = oracle.RenderScene(flat).render(d)
        g = film.cpu().numpy()
        ma, mc = _mean_within(g, c, min_fraction=0.98)
        np.testing.assert_array_equal(g[..., 7], c[..., 7])
        assert mc[..., 1].mean() > 0.01
        # the image means of Y agree within 4 standard errors (pixels are independent estimates: the
        # variance of the image mean is the sum of the pixels' variances of their means / npix^2)
        _, va = R.resolve(g)
        _, vc = R.resolve(c)
        se = np.sqrt((va[..., 1].sum() + vc[..., 1].sum())) / va[..., 1].size
        assert abs(ma[..., 1].mean() - mc[..., 1].mean()) <= 4.0 * se, (ma[..., 1].mean(), mc[..., 1].mean(), se)
        gs.close()
    br.close()


def test_invalid_batches_fail_loudly(cornell):
    gs, cam = cornell
    d = R.render_desc(cam, 8, 8, 1, _tracer(3, 0))
    with pytest.raises(LiarGpuError):
        B.BatchRenderer(default_context(), [(gs, d)], B.make_config(hero=1))     # max_depth 0
    d = R.render_desc(cam, 8, 8, 1, _tracer())
    with pytest.raises(LiarGpuError):
        B.BatchRenderer(default_context(), [(gs, d)], B.make_config(hero=2))
    with pytest.raises(LiarGpuError):
        B.BatchRenderer(default_context(), [(gs, d)], B.make_config(hero=1, max_bounces=4))
    with pytest.raises(LiarGpuError):
        B.BatchRenderer(default_context(), [(gs, d)], B.make_config(hero=1, trace=(64, 8)))
    with pytest.raises(LiarGpuError):
        B.BatchRenderer(default_context(), [(gs, d)], B.make_config(hero=1, shade_blocks_per_sm=3))


def test_autotuner_picks_and_caches(cornell, tmp_path):
    gs, cam = cornell
    entries = [(gs, R.render_desc(cam, 64, 64, 8, _tracer(), seed=1))]
    cache = tmp_path / "tune.json"
    cfg, info = B.tune_batch(default_context(), entries, hero=4, cache=cache, probe_spp=2,
                             trace_shapes=[(128, 16), (256, 8)], wave_sizes=[1 << 14, 1 << 16], shade_grids=[8, 16])
    assert not info["cached"] and cache.exists() and len(info["candidates"]) >= 4
    cfg2, info2 = B.tune_batch(default_context(), entries, hero=4, cache=cache)
    assert info2["cached"] and cfg2.wave_paths == cfg.wave_paths and cfg2.trace.block_size == cfg.trace.block_size
    br = B.BatchRenderer(default_context(), entries, cfg)
    br.launch()
    torch.cuda.synchronize()
    assert br.stats()["paths"] == 64 * 64 * 8
