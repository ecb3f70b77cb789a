"""GPU path tracer (AdjointPhotonTracer estimator) against the CPU restatement of the reference.

Both sides draw the same stratified sample values, so the images agree far inside the workload's
bar (per-pixel means within 3 sigma, sigma from the per-pixel sample variance at matched spp);
they are not bit-identical because the GPU's and the host's sin/cos/exp/log round differently.
"""
import math

import numpy as np
import pytest

import oracle
from liar_b200 import cameras, render as R, scenery, scenes_render, shaders, spectra, textures, tracers
from liar_b200.kernel import default_context

pytestmark = pytest.mark.gpu


def run_both(scene, cam, w, h, spp, max_gen=3, max_depth=8, seed=0):
    tr = tracers.AdjointPhotonTracer()
    tr.maxRayGeneration = max_gen
    tr.maxDepth = max_depth
    flat = R.flatten(scene)
    desc = R.render_desc(cam, w, h, spp, tr, seed=seed)
    gs = R.GpuScene(default_context(), flat)
    g = gs.render(desc)
    stats = gs.stats()
    c = oracle.RenderScene(flat).render(desc)
    return g, c, stats


def within_3_sigma(g, c, min_fraction=0.995):
    mg, vg = R.resolve(g)
    mc, vc = R.resolve(c)
    sig = np.sqrt(vg + vc)
    ok = np.abs(mg[..., :3] - mc[..., :3]) <= 3 * sig + 1e-6 * np.maximum(np.abs(mc[..., :3]), 1.0)
    frac = ok.mean()
    assert frac >= min_fraction, f"only {frac:.4f} of pixel channels within 3 sigma"
    return mg, mc


def test_cornell_matches_oracle():
    scene, cam = scenes_render.cornell_box()
    g, c, stats = run_both(scene, cam, 64, 64, 16)
    assert stats["paths"] == 64 * 64 * 16 and stats["segments"] >= stats["paths"]
    mg, mc = within_3_sigma(g, c)
    np.testing.assert_array_equal(g[..., 7], c[..., 7])          # samples per pixel
    np.testing.assert_array_equal(g[..., 3], c[..., 3])          # alpha: same camera rays, same hits
    assert abs(mg[..., 1].mean() / mc[..., 1].mean() - 1) < 0.01  # image luminance within 1%
    assert mg[..., 1].mean() > 0.01


def test_cornell_workload_at_full_size():
    """The plain path-tracing workload exactly: 256 x 256, 16 spp, Russian roulette from
    generation 3, depth cap 8, seed 0 (the Cornell engine of scenes_render)."""
    e = scenes_render.cornell_engine()
    assert e.sampler.resolution == (256, 256) and e.sampler.samplesPerPixel == 16
    assert (e.tracer.maxRayGeneration, e.tracer.maxDepth, e.seed) == (3, 8, 0)
    g, c, stats = run_both(e.scene, e.camera, 256, 256, 16, max_gen=3, max_depth=8, seed=0)
    assert stats["paths"] == 256 * 256 * 16
    mg, mc = within_3_sigma(g, c)
    np.testing.assert_array_equal(g[..., 7], c[..., 7])
    np.testing.assert_array_equal(g[..., 3], c[..., 3])
    assert abs(mg[..., 1].mean() / mc[..., 1].mean() - 1) < 0.005


def test_cornell_without_depth_cap_and_other_rr_start():
    scene, cam = scenes_render.cornell_box()
    g, c, _ = run_both(scene, cam, 48, 48, 8, max_gen=8, max_depth=0, seed=7)
    within_3_sigma(g, c)


def _box_scene(shader, light_kind="area"):
    floor = scenery.Parallelogram((-2, 0, -2), (4, 0, 0), (0, 0, 4))
    floor.shader = shader
    back = scenery.Parallelogram((-2, 0, 2), (4, 0, 0), (0, 3, 0))
    back.shader = shaders.Lambert(textures.Constant(0.5))
    ball = scenery.Sphere((0, 0.6, 0), 0.6, subdivisions=3)
    ball.shader = shader
    items = [floor, back, ball]
    if light_kind == "area":
        surf = scenery.Parallelogram((-0.5, 2.5, -0.5), (1, 0, 0), (0, 0, 1))
        light = scenery.LightArea(surf)
        light.radiance = spectra.BlackBody(5000, 20)
        items.append(light)
        surf2 = scenery.Parallelogram((1.5, 1.0, -1.0), (0, 0, 0.5), (0, 0.5, 0))
        light2 = scenery.LightArea(surf2)
        light2.radiance = spectra.Spectrum(3.0)
        light2.isDoubleSided = True
        items.append(light2)
    else:
        items.append(scenery.LightSky(textures.Constant(0.8)))
    cam = cameras.PerspectiveCamera()
    cam.position = (0, 1.5, -4)
    cam.lookAt((0, 0.5, 0))
    cam.aspectRatio = 1
    return scenery.List(items), cam


NM = 1e-9


def _cu(kind):
    s = shaders.CookTorrance(textures.Constant(spectra.spd("Cu", "n")), textures.Constant(spectra.spd("Cu", "k")))
    s.roughness = textures.Constant(0.3)
    s.mdf = shaders.MicrofacetTrowbridgeReitz() if kind == "ggx" else shaders.MicrofacetBeckmann()
    return s


def _walter(kind):
    s = shaders.Walter(textures.Constant(1.5))
    s.roughness = textures.Constant(0.2)
    s.mdf = shaders.MicrofacetTrowbridgeReitz() if kind == "ggx" else shaders.MicrofacetBeckmann()
    return s


@pytest.mark.parametrize("name,make", [
    ("lambert", lambda: shaders.Lambert(textures.Constant(spectra.Sampled([400 * NM, 700 * NM], [0.2, 0.9])))),
    ("conductor", lambda: shaders.Conductor(textures.Constant(spectra.spd("Au", "n")),
                                            textures.Constant(spectra.spd("Au", "k")))),
    ("cook_torrance_ggx", lambda: _cu("ggx")),
    ("cook_torrance_beckmann", lambda: _cu("beckmann")),
    ("dielectric_cauchy", lambda: shaders.Dielectric(textures.Constant(spectra.Cauchy(1.5, 0.0042)))),
    ("walter_ggx", lambda: _walter("ggx")),
    ("walter_beckmann", lambda: _walter("beckmann")),
    ("mirror", lambda: shaders.Mirror(textures.Constant(0.9))),
])
def test_bsdf_scenes_match_oracle(name, make):
    scene, cam = _box_scene(make())
    g, c, _ = run_both(scene, cam, 40, 40, 16, max_gen=4, max_depth=10, seed=3)
    mg, mc = within_3_sigma(g, c, min_fraction=0.99)
    assert mg[..., 1].mean() > 0


def test_sky_light_scene_matches_oracle():
    scene, cam = _box_scene(shaders.Lambert(textures.Constant(0.6)), light_kind="sky")
    g, c, _ = run_both(scene, cam, 40, 40, 16, max_gen=4, max_depth=10, seed=5)
    within_3_sigma(g, c, min_fraction=0.99)


def test_white_furnace():
    """Lambert(1) sphere under a constant sky of radiance 1: every sphere pixel converges to Y = 1
    (after the reference's test/white_furnace scene)."""
    scene, cam = scenes_render.white_furnace()
    tr = tracers.AdjointPhotonTracer()
    tr.maxRayGeneration = 2
    flat = R.flatten(scene)
    w = h = 32
    desc = R.render_desc(cam, w, h, 256, tr, seed=11)
    film = R.GpuScene(default_context(), flat).render(desc)
    mean, var = R.resolve(film)
    # pixels whose whole footprint is well inside the sphere's silhouette
    cam_d = cam.flatten()
    ys, xs = np.mgrid[0:h, 0:w]
    sx, sy = (xs + 0.5) / w - 0.5, (ys + 0.5) / h - 0.5
    d = (np.asarray(cam_d["direction"])[None, None] + sx[..., None] * np.asarray(cam_d["right"])
         + sy[..., None] * np.asarray(cam_d["down"]))
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    o = np.asarray(cam_d["position"])
    b = d @ o
    disc = b ** 2 - (o @ o - 1.0)
    inside = disc > 0.25
    assert inside.sum() > 50
    Y = mean[..., 1][inside]
    sig = np.sqrt(var[..., 1][inside])
    z = (Y - 1.0) / np.maximum(sig, 1e-6)
    assert np.mean(np.abs(z) <= 3) > 0.99, f"white furnace: {np.mean(np.abs(z) <= 3):.3f} of pixels within 3 sigma"
    assert abs(Y.mean() - 1.0) < 3 * np.sqrt((var[..., 1][inside]).sum()) / inside.sum() + 0.002


def test_progressive_passes_add_up():
    scene, cam = scenes_render.cornell_box()
    tr = tracers.AdjointPhotonTracer()
    flat = R.flatten(scene)
    gs = R.GpuScene(default_context(), flat)
    film = np.zeros((16, 16, 8), np.float32)
    for k in range(3):
        gs.render(R.render_desc(cam, 16, 16, 4, tr, first_sample=4 * k), film)
    assert (film[..., 7] == 12).all()


def test_render_engine_drop_in():
    """A reference-style script: build, assign, render()."""
    from liar_b200 import RenderEngine, output, samplers
    scene, cam = scenes_render.cornell_box()
    engine = RenderEngine()
    engine.tracer = tracers.AdjointPhotonTracer()
    engine.sampler = samplers.Stratifier((32, 24), 4)
    engine.scene = scene
    engine.camera = cam
    engine.target = output.Display("cornell", (32, 24))
    xyza = engine.render()
    assert xyza.shape == (24, 32, 4)
    assert engine.target.xyza.shape == (24, 32, 4) and engine.target.xyza[..., 1].mean() > 0
