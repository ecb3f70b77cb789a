"""The PhotonMapper on the GPU (csrc/photon_mapper.cu, csrc/direct.cu) against its CPU restatement
(oracle_render.cpp, src/liar/tracers/photon_mapper.cpp). The oracle renders with the maps the GPU
built (their photons are checked against the photon-tracing restatement in
test_photon_trace_gpu.py) and finds each vertex's nearest photons by brute force; both draw the same
camera samples, so images agree within 3 sigma."""
import numpy as np
import pytest
import torch

import oracle
from liar_b200 import recovery, render as R, scenery, scenes_render, shaders, spectra, textures, tracers
from liar_b200.kernel import default_context

pytestmark = pytest.mark.gpu


def _scene():
    """The Cornell box with a glass sphere on the free front-right part of the floor (caustics)."""
    scene, cam = scenes_render.cornell_box()
    glass = scenery.Sphere((4.0, 0.55, 1.2), 0.55, subdivisions=4)
    glass.shader = shaders.Dielectric(textures.Constant(1.5))
    scene.children.append(glass)
    return scene, cam


def _pm(global_size=20_000, direct=True, visualize=False, max_gen=4):
    t = tracers.PhotonMapper()
    t.maxRayGeneration = max_gen
    t.globalMapSize = global_size
    t.isRayTracingDirect = direct
    t.isVisualizingPhotonMap = visualize
    return t


def _close(g, c, min_fraction=0.99, mean_tol=0.02):
    mg, vg = R.resolve(g)
    mc, vc = R.resolve(c)
    sig = np.sqrt(vg + vc)
    ok = np.abs(mg[..., :3] - mc[..., :3]) <= 3 * sig + 1e-5 * np.maximum(np.abs(mc[..., :3]), 1.0)
    assert ok.mean() >= min_fraction, f"only {ok.mean():.4f} of pixel channels within 3 sigma"
    np.testing.assert_array_equal(g[..., 7], c[..., 7])
    assert abs(mg[..., 1].mean() / max(mc[..., 1].mean(), 1e-12) - 1) < mean_tol
    return mg, mc


def _run(tracer, w=32, h=32, spp=4, seed=3):
    scene, cam = _scene()
    flat = R.flatten(scene)
    ctx = default_context()
    gs = R.GpuScene(ctx, flat)
    d = R.render_desc(cam, w, h, spp, tracer, seed=seed)
    g = gs.render(d)
    st = R.photon_mapper_stats(ctx)
    maps = [R.photon_mapper_map(ctx, m) for m in (0, 1)]
    for m in range(2):
        maps[m]["k"] = tracer.estimationSize("global" if m == 0 else "caustic")
    irr = R.photon_mapper_irradiance(ctx)
    st["irradiance"] = irr
    c = oracle.RenderScene(flat).render_pm(d, maps, recovery.device_table(), irradiance=irr)
    return g, c, st, maps


def test_recovery_blends_match_the_host():
    ctx = default_context()
    recovery.set_standard_on(ctx)
    rng = np.random.default_rng(0)
    xyz = rng.uniform(0.0, 1.0, size=(4096, 3)).astype(np.float32)
    xyz[:8] = [[1, 1, 1], [0, 0, 0], [0.2, 0.1, 0.05], [1e-6, 0, 0], [0, 1, 0], [0, 0, 1], [3, 0.1, 0], [0.5, 0.5, 0]]
    d_xyz = torch.from_numpy(xyz).cuda()
    d_idx = torch.empty((4096, 3), dtype=torch.int32, device="cuda")
    d_w = torch.empty((4096, 3), dtype=torch.float32, device="cuda")
    ctx.check(ctx._lib.liar_gpu_recovery_locate_device(ctx.handle, d_xyz.data_ptr(), 4096, d_idx.data_ptr(),
                                                       d_w.data_ptr(), None))
    torch.cuda.synchronize()
    gi, gw = d_idx.cpu().numpy(), d_w.cpu().numpy()
    rec = recovery.standard()
    lam = np.linspace(380e-9, 720e-9, 9, dtype=np.float32)
    t = recovery.device_table()
    for i in range(4096):
        loc = rec.locate(xyz[i])
        if loc is None:
            assert (gi[i] == -1).all() and (gw[i] == 0).all()
            continue
        # the same blend (the triangle's order of corners may differ): compare the spectra it gives
        for w in lam[::4]:
            host = rec.recover(xyz[i], float(w))
            k = int(np.searchsorted(t["wavelengths"], w, side="right"))
            tt = (w - t["wavelengths"][k - 1]) / (t["wavelengths"][k] - t["wavelengths"][k - 1])
            v0 = sum(gw[i, j] * t["spectra"][gi[i, j], k - 1] for j in range(3) if gi[i, j] >= 0)
            v1 = sum(gw[i, j] * t["spectra"][gi[i, j], k] for j in range(3) if gi[i, j] >= 0)
            assert abs(v0 + tt * (v1 - v0) - host) <= 1e-4 * max(1.0, abs(host)) + 1e-6 * xyz[i].sum()


def test_photon_mapper_matches_oracle():
    g, c, st, maps = _run(_pm())
    assert st["valid"] and st["emitted"] > 0
    # fillPhotonMaps stops with the emission that fills the global map: at most one photon path more
    assert 20_000 <= st["global"] <= 20_000 + 4 and st["caustic"] > 0
    assert st["radius"][0] > 0 and st["radius"][1] > 0
    # the powers are XYZ scaled by 1 / photons shot, every one with a recovery blend
    assert (maps[0]["blend_idx"] >= -1).all() and (maps[0]["blend_w"].sum(axis=1) > 0).mean() > 0.99
    mg, _ = _close(g, c)
    assert mg[..., 1].mean() > 1e-3


def test_photon_mapper_without_traced_direct_light():
    g, c, _, _ = _run(_pm(direct=False), seed=5)
    _close(g, c)


def test_visualised_photon_map():
    g, c, _, _ = _run(_pm(visualize=True), w=24, h=24, spp=2, seed=7)
    mg, _ = _close(g, c)
    assert mg[..., 1].mean() > 1e-3


def _fg(rays=8, ratio=0.25, secondary=1, global_size=20_000):
    t = _pm(global_size=global_size)
    t.numFinalGatherRays = rays
    t.ratioPrecomputedIrradiance = ratio
    t.numSecondaryGatherRays = secondary
    return t


def test_final_gathering_matches_oracle():
    """numFinalGatherRays > 0: camera (and specular-chain) diffuse vertices gather the indirect
    light with BSDF-sampled rays evaluated from the precomputed irradiance map, with a secondary
    gather and low-quality direct light where a gather hit is closer than the estimate's radius."""
    g, c, st, maps = _run(_fg(), w=24, h=24, spp=2, seed=9)
    irr = st["irradiance"]
    # with final gathering every diffuse hit is a global photon, a quarter of them irradiance points
    assert 20_000 <= st["global"] <= 20_004
    assert 0.2 * st["global"] < len(irr["position"]) < 0.3 * st["global"]
    assert (irr["r2"] > 0).mean() > 0.99 and np.allclose(np.linalg.norm(irr["normal"], axis=1), 1, atol=1e-3)
    mg, _ = _close(g, c)
    assert mg[..., 1].mean() > 1e-3


def test_final_gathering_without_irradiance_map_or_secondary_rays():
    g, c, st, _ = _run(_fg(rays=6, ratio=0.0, secondary=0), w=20, h=20, spp=2, seed=11)
    assert len(st["irradiance"]["position"]) == 0
    _close(g, c)


def test_maps_are_kept_for_the_same_scene_and_settings():
    scene, cam = _scene()
    flat = R.flatten(scene)
    ctx = default_context()
    gs = R.GpuScene(ctx, flat)
    t = _pm(global_size=5_000)
    gs.render(R.render_desc(cam, 8, 8, 1, t, seed=1))
    a = R.photon_mapper_map(ctx, 0)
    gs.render(R.render_desc(cam, 8, 8, 1, t, seed=1, first_sample=1))
    b = R.photon_mapper_map(ctx, 0)
    np.testing.assert_array_equal(a["position"], b["position"])
    t.setEstimationSize("global", 20)
    gs.render(R.render_desc(cam, 8, 8, 1, t, seed=1))
    assert R.photon_mapper_stats(ctx)["global"] >= 5_000


def test_photon_mapper_agrees_with_path_tracing_on_average():
    """Density estimation blurs, but in the diffuse box the mean luminance of the lit surfaces stays
    within a few percent of the unbiased path tracer's (the light itself, a sub-pixel emitter far
    brighter than the rest, is left out of the comparison)."""
    scene, cam = scenes_render.cornell_box()
    flat = R.flatten(scene)
    gs = R.GpuScene(default_context(), flat)
    pm = gs.render(R.render_desc(cam, 48, 48, 16, _pm(global_size=200_000, max_gen=8), seed=2))
    pt_tracer = tracers.AdjointPhotonTracer()
    pt_tracer.maxRayGeneration = 8
    pt = gs.render(R.render_desc(cam, 48, 48, 256, pt_tracer, seed=2))
    a, _ = R.resolve(pm)
    b, _ = R.resolve(pt)
    lit = (a[..., 1] < 2.0) & (b[..., 1] < 2.0)
    assert lit.mean() > 0.95
    ya, yb = a[..., 1][lit].mean(), b[..., 1][lit].mean()
    assert abs(ya / yb - 1) < 0.1, (ya, yb)


def test_final_gathering_agrees_with_path_tracing_on_average():
    scene, cam = scenes_render.cornell_box()
    flat = R.flatten(scene)
    gs = R.GpuScene(default_context(), flat)
    t = _fg(rays=16, global_size=100_000)
    t.maxRayGeneration = 8
    pm = gs.render(R.render_desc(cam, 40, 40, 4, t, seed=4))
    pt_tracer = tracers.AdjointPhotonTracer()
    pt_tracer.maxRayGeneration = 8
    pt = gs.render(R.render_desc(cam, 40, 40, 256, pt_tracer, seed=4))
    a, _ = R.resolve(pm)
    b, _ = R.resolve(pt)
    lit = (a[..., 1] < 2.0) & (b[..., 1] < 2.0)
    ya, yb = a[..., 1][lit].mean(), b[..., 1][lit].mean()
    assert abs(ya / yb - 1) < 0.1, (ya, yb)


def test_caustics_quality_matches_oracle():
    """causticsQuality 4: the global map is filled at storage probability 1/4 (four times the
    emissions), every caustic photon is kept, and the maps' powers are divided by their
    probabilities; the render agrees with the oracle over the same maps, and its global map is the
    requested size."""
    t = _pm(global_size=8_000)
    t.causticsQuality = 4.0
    g, c, st, maps = _run(t, w=32, h=32, spp=4, seed=6)
    _close(g, c)
    assert st["global"] == 8_000
    t1 = _pm(global_size=8_000)
    _, _, st1, _ = _run(t1, w=8, h=8, spp=1, seed=6)
    assert st["emitted"] > 2.5 * st1["emitted"]
    assert st["caustic"] > 2.0 * st1["caustic"]


def test_unsupported_settings_fail_loudly():
    scene, cam = _scene()
    t = _pm()
    t.setEstimationSize("caustic", 100)
    gs = R.GpuScene(default_context(), R.flatten(scene))
    from liar_b200._native import LiarGpuError
    with pytest.raises(LiarGpuError):
        gs.render(R.render_desc(cam, 8, 8, 1, t))
