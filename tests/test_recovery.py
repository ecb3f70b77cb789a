"""Tristimulus-to-spectrum recovery (spectra/recovery_meng_simon.cpp) and the reference's rgb()
(kernel/rgb_space.cpp): the recovered spectrum reproduces its XYZ under the standard observer,
white recovers the flat spectrum, and a recovered colour renders like its sampled spectrum."""
import numpy as np
import pytest

import oracle
from liar_b200 import _tables, recovery, render as R, rgb, scenes_render, shaders, spectra, textures, tracers


def _tristimulus(values_at):
    o = _tables.observer().astype(np.float64)
    w = o[:, 0]
    v = values_at(w)
    dw = np.gradient(w)
    y = np.sum(o[:, 2] * dw)
    return np.array([np.sum(v * o[:, k] * dw) for k in (1, 2, 3)]) / y


@pytest.mark.parametrize("c", [(0.7, 0.1, 0.1), (0.1, 0.7, 0.1), (0.1, 0.1, 0.7), (0.2, 0.5, 0.3), (0.9, 0.8, 0.1)])
def test_recovered_spectrum_reproduces_its_tristimulus(c):
    s = rgb(*c)
    np.testing.assert_allclose(_tristimulus(s), s.xyz, rtol=0.02, atol=2e-3)


def test_white_is_flat_and_black_is_zero():
    w = np.linspace(380e-9, 720e-9, 35)
    np.testing.assert_allclose(rgb(1, 1, 1)(w), 1.0, atol=1e-3)
    assert np.all(rgb(0, 0, 0)(w) == 0)
    assert rgb((0.5, 0.5, 0.5)).xyz == rgb(0.5, 0.5, 0.5).xyz


def test_srgb_primaries_adapted_to_e():
    """The sRGB white (1, 1, 1) maps to the white of illuminant E, X = Y = Z = 1 (Bradford adapted)."""
    np.testing.assert_allclose(recovery.sRGB.toXYZ((1.0, 1.0, 1.0)), (1.0, 1.0, 1.0), atol=1e-4)
    # the gamma: rgb(0.5) is 0.5^2.2 of white
    np.testing.assert_allclose(recovery.sRGB.toXYZ((0.5, 0.5, 0.5))[1], 0.5 ** 2.2, rtol=1e-5)


def test_blend_weights_sum_to_the_colour_sum():
    rec = recovery.standard()
    for xyz in [(0.2, 0.1, 0.05), (0.3, 0.3, 0.3), (0.05, 0.2, 0.6)]:
        idx, w = rec.locate(xyz)
        assert np.isclose(w.sum(), sum(xyz), rtol=1e-5)
        assert all(wi >= -1e-6 for wi in w)
    assert rec.locate((0.0, 0.0, 0.0)) is None


def test_recovered_colour_renders_as_its_table():
    """An rgb() Lambert wall flattens to the recovered table; the oracle renders the wall with the
    same value as a Sampled spectrum built from the recovery by hand."""
    scene, cam = scenes_render.cornell_box()
    c = rgb(0.7, 0.1, 0.1)
    ws, vs, mx = recovery.standard().sampled(c.xyz)
    by_hand = spectra.Sampled(ws.tolist(), vs.tolist())
    t = tracers.AdjointPhotonTracer()
    t.maxRayGeneration = 2
    t.maxDepth = 4
    images = []
    for spec in (c, by_hand):
        scene.children[5].shader = shaders.Lambert(textures.Constant(spec))  # the red (left) wall
        flat = R.flatten(scene)
        d = R.render_desc(cam, 16, 16, 4, t, seed=1)
        images.append(oracle.RenderScene(flat).render(d))
    # the reflectance bound of the recovered colour is the blend of maxima (<= 1 here): same image
    assert mx <= 1.0
    np.testing.assert_array_equal(images[0], images[1])
