"""The film on the CPU restatement: reconstruction filters (output/filter_triangle.cpp,
output/filter_mitchell.cpp) and the sample luminance clamp (output/raster.cpp:572-575)."""
import math

import numpy as np
import pytest

import oracle
from liar_b200 import output, render as R, scenes_render, tracers


def _render(scene, cam, w, h, spp, **film):
    t = tracers.AdjointPhotonTracer()
    t.maxRayGeneration = 64
    t.maxDepth = 64
    d = R.render_desc(cam, w, h, spp, t, seed=3, **film)
    return oracle.RenderScene(R.flatten(scene)).render(d)


@pytest.mark.parametrize("film", [dict(filter=R.FILTER_TRIANGLE, filter_param=1.5),
                                  dict(filter=R.FILTER_TRIANGLE, filter_param=1.0),
                                  dict(filter=R.FILTER_MITCHELL)])
def test_filtered_white_furnace_stays_one(film):
    """Normalised by the sum of the weights, a filtered pixel keeps the expectation of its
    neighbourhood: on the unit-albedo sphere under a unit sky every such pixel converges to Y = 1."""
    scene, cam = scenes_render.white_furnace()
    f = _render(scene, cam, 24, 24, 48, **film)
    box = _render(scene, cam, 24, 24, 48)
    mb, _ = R.resolve(box)
    m, v = R.resolve(f)
    # pixels whose whole filter footprint lies well inside the unit sphere's silhouette
    cd = cam.flatten()
    ys, xs = np.mgrid[0:24, 0:24]
    sx, sy = (xs + 0.5) / 24 - 0.5, (ys + 0.5) / 24 - 0.5
    dirs = (np.asarray(cd["direction"])[None, None] + sx[..., None] * np.asarray(cd["right"])
            + sy[..., None] * np.asarray(cd["down"]))
    dirs /= np.linalg.norm(dirs, axis=-1, keepdims=True)
    o = np.asarray(cd["position"])
    inner = (dirs @ o) ** 2 - (o @ o - 1.0) > 0.5
    assert inner.sum() > 40
    y = m[..., 1][inner]
    se = math.sqrt(float(mb[..., 1][inner].var()) / inner.sum() + 1e-6)
    assert abs(y.mean() - 1.0) < max(6 * se, 0.03)
    if film.get("filter_param") != 1.5:
        # the weights: a sample gives its footprint a total weight of 1 (the unit triangle and
        # Mitchell-Netravali with B + 2C = 1 are partitions of unity), less what falls outside
        n = 24 * 24 * 48
        tot = float(f[..., 7].sum())
        assert 0.85 * n < tot < 1.05 * n


def test_triangle_weights_are_the_reference_kernel():
    """Width 0.5: only the sample's own pixel has weight, (0.5 - |dx|)(0.5 - |dy|) <= 1/4."""
    scene, cam = scenes_render.cornell_box()
    f = _render(scene, cam, 16, 16, 8, filter=R.FILTER_TRIANGLE, filter_param=0.5)
    w = f[..., 7]
    assert (w > 0).all() and (w <= 8 * 0.25 + 1e-6).all()
    box = _render(scene, cam, 16, 16, 8)
    np.testing.assert_array_equal(f[..., 3] > 0, box[..., 3] > 0)


def test_luminance_clamp():
    scene, cam = scenes_render.cornell_box()
    free = _render(scene, cam, 16, 16, 8)
    m0, _ = R.resolve(free)
    cap = float(np.percentile(m0[..., 1], 30))
    clamped = _render(scene, cam, 16, 16, 8, max_sample_luminance=cap)
    m, _ = R.resolve(clamped)
    assert (m[..., 1] <= cap * (1 + 1e-5)).all()
    assert m[..., 1].mean() < m0[..., 1].mean()
    # chromaticity of every sample is kept: X/Y of the clamped pixel stays within the free pixel's range
    assert np.all(np.isfinite(m))


def test_render_targets_select_the_film():
    img = output.Image("x.npy", (8, 8))
    assert output.film_settings(img) == {"filter": 0, "filter_param": 0.0, "max_sample_luminance": 0.0}
    img.maxSampleLuminance = 5.0
    assert output.film_settings(output.FilterMitchell(img)) == {"filter": 2, "filter_param": 1.0 / 3.0,
                                                                "max_sample_luminance": 5.0}
    assert output.film_settings(output.FilterTriangle(img, 2.0))["filter_param"] == 2.0
    with pytest.raises(ValueError):
        output.film_settings(output.FilterTriangle(img, 0.0))
