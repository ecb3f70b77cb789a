"""The reference's Cornell box example scripts rendered on the GPU: the fixtures hold what
examples/cornell_box/direct_lighting.py and photon_mapper_classic.py, run unchanged through the
``liar`` package (tests/golden/make_example_scenes.py), asked the engine to render: the measured
Cornell box spectra of liar.tools.cornell_box, DirectLighting, and the classic PhotonMapper with
final gathering and an unjittered stratifier. Each image must agree with the oracle's
restatement within 3 sigma. Also: the samplers' patterns against the oracle, and cancellation
through the C ABI's cancel flag."""
import ctypes as C
import sys
import threading
import time
from pathlib import Path

import numpy as np
import pytest

import oracle
from liar_b200 import recovery, render as R, samplers, scenes_render, tracers
from liar_b200._native import LiarGpuError
from liar_b200.kernel import default_context

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE / "golden"))
import scene_io  # noqa: E402

pytestmark = pytest.mark.gpu


def _close(g, c, min_fraction=0.99, mean_tol=0.02):
    mg, vg = R.resolve(g)
    mc, vc = R.resolve(c)
    sig = np.sqrt(vg + vc)
    ok = np.abs(mg[..., :3] - mc[..., :3]) <= 3 * sig + 1e-5 * np.maximum(np.abs(mc[..., :3]), 1.0)
    assert ok.mean() >= min_fraction, f"only {ok.mean():.4f} of pixel channels within 3 sigma"
    np.testing.assert_array_equal(g[..., 7], c[..., 7])  # every pixel got its samples
    assert abs(mg[..., 1].mean() / max(mc[..., 1].mean(), 1e-12) - 1) < mean_tol
    return mg, mc


def test_direct_lighting_example_renders_like_the_oracle():
    flat, desc, _ = scene_io.load(HERE / "golden" / "example_direct_lighting.npz")
    assert desc.tracer == 1 and desc.sampler == 0
    g = R.GpuScene(default_context(), flat).render(desc)
    c = oracle.RenderScene(flat).render(desc)
    mg, _ = _close(g, c, min_fraction=0.995, mean_tol=0.01)
    assert mg[..., 1].mean() > 0.01


def test_photon_mapper_classic_example_renders_like_the_oracle():
    flat, desc, _ = scene_io.load(HERE / "golden" / "example_photon_mapper_classic.npz")
    assert desc.tracer == 2 and desc.sampler == samplers.LIAR_SAMPLER_NOT_JITTERED
    assert desc.photon_mapper.final_gather_rays == 16
    ctx = default_context()
    g = R.GpuScene(ctx, flat).render(desc)
    maps = [R.photon_mapper_map(ctx, m) for m in (0, 1)]
    for m in range(2):
        maps[m]["k"] = int(desc.photon_mapper.estimation_size[m])
    irr = R.photon_mapper_irradiance(ctx)
    assert len(maps[0]["position"]) > 1000 and len(irr["position"]) > 0
    c = oracle.RenderScene(flat).render_pm(desc, maps, recovery.device_table(), irradiance=irr)
    mg, _ = _close(g, c)
    assert mg[..., 1].mean() > 0.01


@pytest.mark.parametrize("mode", [samplers.LIAR_SAMPLER_STRATIFIER, samplers.LIAR_SAMPLER_NOT_JITTERED,
                                  samplers.LIAR_SAMPLER_LATIN_HYPERCUBE,
                                  samplers.LIAR_SAMPLER_LATIN_HYPERCUBE | samplers.LIAR_SAMPLER_NOT_JITTERED])
def test_sampler_patterns_render_like_the_oracle(mode):
    scene, cam = scenes_render.cornell_box()
    flat = R.flatten(scene)
    t = tracers.AdjointPhotonTracer()
    t.maxRayGeneration = 3
    t.maxDepth = 8
    desc = R.render_desc(cam, 48, 48, 9, t, seed=5, sampler=mode)
    g = R.GpuScene(default_context(), flat).render(desc)
    c = oracle.RenderScene(flat).render(desc)
    _close(g, c, min_fraction=0.99, mean_tol=0.02)
    np.testing.assert_array_equal(g[..., 3], c[..., 3])  # camera rays (alpha) are identical


def test_cancel_flag_stops_a_render_and_leaves_the_context_usable():
    ctx = default_context()
    scene, cam = scenes_render.cornell_box()
    gs = R.GpuScene(ctx, R.flatten(scene))
    t = tracers.AdjointPhotonTracer()
    small = R.render_desc(cam, 32, 32, 4, t, seed=1)
    flag = C.c_int32(1)
    ctx.set_cancel_flag(flag)
    try:
        with pytest.raises(LiarGpuError) as err:
            gs.render(small)
        assert err.value.code == -7  # LIAR_ERR_CANCELLED, before any wave
        # raised from another thread while a long render runs (1024 waves of 64k paths, each with
        # a host wait per bounce: far longer than the timer)
        flag.value = 0
        big = R.render_desc(cam, 1024, 1024, 64, t, seed=2, wave_paths=1 << 16)
        timer = threading.Timer(0.05, lambda: setattr(flag, "value", 1))
        t0 = time.perf_counter()
        timer.start()
        with pytest.raises(LiarGpuError) as err:
            gs.render(big)
        elapsed = time.perf_counter() - t0
        timer.join()
        assert err.value.code == -7
        assert elapsed < 5.0
    finally:
        ctx.set_cancel_flag(None)
    # the context renders normally afterwards, and like the oracle
    g = gs.render(small)
    c = oracle.RenderScene(R.flatten(scene)).render(small)
    _close(g, c, min_fraction=0.99, mean_tol=0.03)


def test_cancel_flag_stops_direct_lighting():
    ctx = default_context()
    scene, cam = scenes_render.cornell_box()
    gs = R.GpuScene(ctx, R.flatten(scene))
    flag = C.c_int32(1)
    ctx.set_cancel_flag(flag)
    try:
        with pytest.raises(LiarGpuError) as err:
            gs.render(R.render_desc(cam, 16, 16, 1, tracers.DirectLighting(), seed=1))
        assert err.value.code == -7
    finally:
        ctx.set_cancel_flag(None)
    gs.render(R.render_desc(cam, 16, 16, 1, tracers.DirectLighting(), seed=1))
