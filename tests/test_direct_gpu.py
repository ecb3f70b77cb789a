"""DirectLighting on the GPU (csrc/direct.cu) against its CPU restatement (oracle_render.cpp), which
follows src/liar/tracers/direct_lighting.cpp and RayTracer::estimateLightContribution
(src/liar/kernel/ray_tracer.cpp:188-276). Both sides draw the same sample values, so the images
agree far inside 3 sigma; they differ only where the GPU's and the host's float functions round
differently."""
import numpy as np
import pytest

import oracle
from liar_b200 import cameras, render as R, scenery, scenes_render, shaders, spectra, textures, tracers
from liar_b200.kernel import default_context

pytestmark = pytest.mark.gpu


def _tracer(max_gen=8, secondary=1, glossy=True):
    t = tracers.DirectLighting()
    t.maxRayGeneration = max_gen
    t.numberOfSecondaryLightSamples = secondary
    t.traceGlossy = glossy
    return t


def run_both(scene, cam, w, h, spp, tracer, seed=0):
    flat = R.flatten(scene)
    desc = R.render_desc(cam, w, h, spp, tracer, seed=seed)
    gs = R.GpuScene(default_context(), flat)
    g = gs.render(desc)
    stats = gs.stats()
    c = oracle.RenderScene(flat).render(desc)
    return g, c, stats


def close(g, c, min_fraction=0.995, mean_tol=0.01):
    mg, vg = R.resolve(g)
    mc, vc = R.resolve(c)
    sig = np.sqrt(vg + vc)
    ok = np.abs(mg[..., :3] - mc[..., :3]) <= 3 * sig + 1e-5 * np.maximum(np.abs(mc[..., :3]), 1.0)
    assert ok.mean() >= min_fraction, f"only {ok.mean():.4f} of pixel channels within 3 sigma"
    np.testing.assert_array_equal(g[..., 7], c[..., 7])
    np.testing.assert_array_equal(g[..., 3], c[..., 3])
    assert abs(mg[..., 1].mean() / max(mc[..., 1].mean(), 1e-12) - 1) < mean_tol
    return mg, mc


def test_cornell_direct_lighting():
    """16 light and 16 BSDF samples per vertex on the Cornell box (all Lambert: direct light only)."""
    scene, cam = scenes_render.cornell_box()
    g, c, st = run_both(scene, cam, 48, 48, 4, _tracer(), seed=3)
    mg, mc = close(g, c)
    assert mg[..., 1].mean() > 0.01
    assert st["paths"] == 48 * 48 * 4
    # camera rays only (no specular surfaces): one segment per sample, all of them hit the box
    assert st["segments"] == st["paths"]


def _showcase(light="area"):
    """Lambert floor and wall, a mirror, a glass, a GGX copper and a Walter sphere; area, point and
    sky lights."""
    floor = scenery.Parallelogram((-3, 0, -3), (0, 0, 6), (6, 0, 0))
    floor.shader = shaders.Lambert(textures.Constant(0.6))
    back = scenery.Parallelogram((-3, 0, 2.5), (6, 0, 0), (0, 3, 0))
    back.shader = shaders.Lambert(textures.Constant(spectra.Sampled([380e-9, 550e-9, 720e-9], [0.2, 0.5, 0.8])))
    mirror = scenery.Sphere((-1.6, 0.5, 0.5), 0.5, subdivisions=3)
    mirror.shader = shaders.Mirror(textures.Constant(0.9))
    glass = scenery.Sphere((-0.4, 0.5, -0.3), 0.5, subdivisions=3)
    glass.shader = shaders.Dielectric(textures.Constant(spectra.Cauchy(1.5, 0.0042)))
    cu = shaders.CookTorrance(textures.Constant(spectra.spd("Cu", "n")), textures.Constant(spectra.spd("Cu", "k")))
    cu.mdf = shaders.MicrofacetTrowbridgeReitz()
    cu.roughness = textures.Constant(0.3)
    metal = scenery.Sphere((0.8, 0.5, 0.4), 0.5, subdivisions=3)
    metal.shader = cu
    frosted = shaders.Walter(textures.Constant(1.5))
    frosted.roughness = textures.Constant(0.2)
    ball = scenery.Sphere((1.9, 0.4, -0.6), 0.4, subdivisions=3)
    ball.shader = frosted
    items = [floor, back, mirror, glass, metal, ball]
    if light in ("area", "all"):
        lamp = scenery.LightArea(scenery.Parallelogram((-0.5, 2.8, -0.5), (1, 0, 0), (0, 0, 1)))
        lamp.radiance = spectra.BlackBody(5000, 15)
        lamp.numberOfEmissionSamples = 4
        items.append(lamp)
        side = scenery.LightArea(scenery.Parallelogram((2.8, 0.5, -1.0), (0, 0, 0.6), (0, 0.6, 0)))
        side.radiance = spectra.Spectrum(4.0)
        side.isDoubleSided = True
        side.numberOfEmissionSamples = 2
        items.append(side)
    if light in ("point", "all"):
        items.append(scenery.LightPoint((1.0, 2.0, -1.5), spectra.BlackBody(3000, 6)))
    if light in ("sky", "all"):
        items.append(scenery.LightSky(textures.Constant(0.3)))
    cam = cameras.PerspectiveCamera()
    cam.position = (0, 1.5, -4.5)
    cam.sky = (0, 1, 0)
    cam.lookAt((0, 0.5, 0))
    cam.aspectRatio = 4 / 3
    return scenery.List(items), cam


@pytest.mark.parametrize("light", ["area", "point", "sky", "all"])
def test_specular_glossy_scene(light):
    scene, cam = _showcase(light)
    g, c, st = run_both(scene, cam, 40, 30, 4, _tracer(), seed=11)
    mg, _ = close(g, c, min_fraction=0.99, mean_tol=0.02)
    assert mg[..., 1].mean() > 1e-3
    assert st["segments"] > st["paths"]  # specular and glossy children were traced


def test_secondary_samples_and_no_glossy():
    scene, cam = _showcase("all")
    g, c, _ = run_both(scene, cam, 32, 24, 2, _tracer(max_gen=4, secondary=3, glossy=False), seed=5)
    close(g, c, min_fraction=0.99, mean_tol=0.02)


def test_generation_cap_zero_is_direct_only():
    """maxRayGeneration 0: camera vertices only (RayTracer::castRay stops beyond it)."""
    scene, cam = _showcase("area")
    g, c, st = run_both(scene, cam, 32, 24, 2, _tracer(max_gen=0), seed=2)
    close(g, c)
    assert st["segments"] == st["paths"]
