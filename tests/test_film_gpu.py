"""The GPU film with the reference's reconstruction filters (output/filter_triangle.cpp,
output/filter_mitchell.cpp) and sample clamp (output/raster.cpp:572-575), against the CPU
restatement: both draw the same samples and give them the same weights, so the weight sums agree
to float rounding (only the order of the additions differs) and the images within 3 sigma."""
import numpy as np
import pytest
import torch

import oracle
from liar_b200 import batch as B, guiding as GD, render as R, scenes_render, tracers
from liar_b200._native import LiarGpuError
from liar_b200.kernel import default_context

pytestmark = pytest.mark.gpu

FILMS = [dict(filter=R.FILTER_TRIANGLE, filter_param=1.5), dict(filter=R.FILTER_MITCHELL),
         dict(filter=R.FILTER_MITCHELL, filter_param=0.5, max_sample_luminance=0.05),
         dict(max_sample_luminance=0.02)]


def _pt(max_gen=3, max_depth=8):
    t = tracers.AdjointPhotonTracer()
    t.maxRayGeneration = max_gen
    t.maxDepth = max_depth
    return t


def _check(g, c, min_fraction=0.99):
    np.testing.assert_allclose(g[..., 7], c[..., 7], rtol=2e-5, atol=1e-5)
    np.testing.assert_allclose(g[..., 3], c[..., 3], rtol=2e-5, atol=1e-5)
    mg, vg = R.resolve(g)
    mc, vc = R.resolve(c)
    sig = np.sqrt(vg + vc)
    ok = np.abs(mg[..., :3] - mc[..., :3]) <= 3 * sig + 1e-5 * np.maximum(np.abs(mc[..., :3]), 1.0)
    assert ok.mean() >= min_fraction, f"only {ok.mean():.4f} of pixel channels within 3 sigma"
    assert abs(mg[..., 1].mean() / mc[..., 1].mean() - 1) < 0.02
    return mg, mc


@pytest.mark.parametrize("film", FILMS)
def test_path_tracer_film_matches_oracle(film):
    scene, cam = scenes_render.cornell_box()
    flat = R.flatten(scene)
    d = R.render_desc(cam, 40, 40, 8, _pt(), seed=4, **film)
    g = R.GpuScene(default_context(), flat).render(d)
    c = oracle.RenderScene(flat).render(d)
    mg, _ = _check(g, c)
    if film.get("max_sample_luminance") and not film.get("filter"):
        assert (mg[..., 1] <= film["max_sample_luminance"] * (1 + 1e-5)).all()


def test_direct_lighting_film_matches_oracle():
    scene, cam = scenes_render.cornell_box()
    flat = R.flatten(scene)
    d = R.render_desc(cam, 32, 32, 2, tracers.DirectLighting(), seed=6, filter=R.FILTER_MITCHELL)
    _check(R.GpuScene(default_context(), flat).render(d), oracle.RenderScene(flat).render(d))


def _device_film(d):
    return torch.zeros((d.height, d.width, 8), dtype=torch.float32, device="cuda:0")


def test_guided_and_batched_films_match_the_single_render():
    """The guided renderer with the guide off and a one-wavelength batch item draw the single
    renderer's samples: with a filter their films agree with its film to rounding."""
    scene, cam = scenes_render.cornell_box()
    flat = R.flatten(scene)
    gs = R.GpuScene(default_context(), flat)
    d = R.render_desc(cam, 36, 28, 6, _pt(), seed=2, filter=R.FILTER_TRIANGLE, filter_param=2.0,
                      max_sample_luminance=0.1)
    ref = _device_film(d)
    gs.render_device(d, ref.data_ptr())
    g = GD.Guide(default_context(), GD.scene_bounds(flat), guide_probability=0.0)
    guided = _device_film(d)
    g.render(gs, d, guided.data_ptr(), train=False)
    br = B.BatchRenderer(default_context(), [(gs, d)], B.make_config(hero=1))
    br.launch()
    torch.cuda.synchronize()
    r = ref.cpu().numpy()
    scale = max(float(np.abs(r[..., :7]).max()), 1e-6)
    for other in (guided.cpu().numpy(), br.films[0].cpu().numpy()):
        np.testing.assert_allclose(other[..., :8], r[..., :8], rtol=2e-5, atol=2e-6 * scale)
    br.close()
    g.close()


def test_invalid_film_settings_fail_loudly():
    scene, cam = scenes_render.cornell_box()
    gs = R.GpuScene(default_context(), R.flatten(scene))
    for bad in (dict(filter=7), dict(filter=R.FILTER_TRIANGLE, filter_param=-1.0),
                dict(filter=R.FILTER_TRIANGLE, filter_param=20.0), dict(max_sample_luminance=-1.0)):
        with pytest.raises(LiarGpuError):
            gs.render(R.render_desc(cam, 8, 8, 1, _pt(), **bad))
