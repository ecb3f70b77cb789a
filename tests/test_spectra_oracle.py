"""CPU checks of the spectral restatement: the reference's Sampled known answer
(tests/golden/sampled_resample.json from test/test_spectrum.cpp:256-278), blackbody and Cauchy
closed forms, the observer's normalisation and sampling pdf, and the oracle's path tracer
(white furnace, light emission) on small cases."""
import ctypes as C
import json
import math
from pathlib import Path

import numpy as np
import pytest

import oracle
from liar_b200 import _tables, render as R, scenery, scenes_render, shaders, spectra, textures, tracers

GOLD = json.loads((Path(__file__).parent / "golden" / "sampled_resample.json").read_text())


def test_python_sampled_resample_known_answer():
    s = spectra.Sampled(GOLD["sampled_wavelengths"], GOLD["sampled_values"])
    r = s.resample(GOLD["resample_wavelengths"])
    np.testing.assert_allclose(r.wavelengths, GOLD["resample_wavelengths"], atol=GOLD["tolerance"])
    np.testing.assert_allclose(r.values, GOLD["expected_values"], atol=GOLD["tolerance"])


def _scene_with(spec_list):
    """A one-triangle scene whose spectrum table holds spec_list (via Lambert shaders)."""
    items = []
    for k, sp in enumerate(spec_list):
        t = scenery.Triangle((k, 0, 0), (k + 1, 0, 0), (k, 1, 0))
        t.shader = shaders.Lambert(textures.Constant(sp))
        items.append(t)
    return R.flatten(scenery.List(items))


def _eval(flat, idx, w, reflectant=False):
    L = oracle.lib()
    L.oracle_spectrum_eval.restype = C.c_float
    L.oracle_spectrum_eval.argtypes = [C.c_void_p, C.c_int, C.c_float, C.c_int]
    rs = oracle.RenderScene(flat)
    return L.oracle_spectrum_eval(rs.h, idx, w, int(reflectant)), rs


def test_oracle_sampled_matches_known_answer():
    s = spectra.Sampled(GOLD["sampled_wavelengths"], GOLD["sampled_values"])
    flat = _scene_with([s])
    for w, v in zip(GOLD["resample_wavelengths"], GOLD["expected_values"]):
        got, _ = _eval(flat, 0, w)
        assert abs(got - v) <= GOLD["tolerance"], (w, got, v)


def test_oracle_reflectant_rescale_and_clamp():
    s = spectra.Sampled([400e-9, 700e-9], [0.5, 2.0])  # max 2 -> divided by 2 when reflectant
    flat = _scene_with([s, spectra.Spectrum(1.7)])
    assert abs(_eval(flat, 0, 550e-9, True)[0] - 0.625) < 1e-6
    assert abs(_eval(flat, 0, 550e-9, False)[0] - 1.25) < 1e-6
    assert _eval(flat, 1, 550e-9, True)[0] == 1.0
    assert abs(_eval(flat, 1, 550e-9, False)[0] - 1.7) < 1e-6


def test_oracle_blackbody_and_cauchy():
    bb = spectra.BlackBody(2856.0, 3.0)
    ca = spectra.Cauchy(1.5, 0.0042)
    flat = _scene_with([bb, ca])
    for w in (380e-9, 500e-9, 760e-9):
        assert abs(_eval(flat, 0, w)[0] / float(bb(w)) - 1) < 1e-4
        assert abs(_eval(flat, 1, w)[0] - float(ca(w))) < 1e-6
    assert abs(_eval(flat, 0, bb.peakWavelength)[0] - 3.0) < 1e-4  # normalised at the peak


def test_observer_normalisation_and_pdf():
    flat = _scene_with([spectra.Spectrum(1.0)])
    rs = oracle.RenderScene(flat)
    L = oracle.lib()
    L.oracle_observer_sample.restype = C.c_float
    L.oracle_observer_sample.argtypes = [C.c_void_p, C.c_float, C.c_void_p, C.c_void_p]
    us = (np.arange(4096) + 0.5) / 4096
    Ys = []
    for u in us:
        pdf = C.c_float()
        xyz = (C.c_float * 3)()
        w = L.oracle_observer_sample(rs.h, float(u), C.byref(pdf), xyz)
        assert pdf.value > 0 and 360e-9 <= w <= 830e-9
        Ys.append(xyz[1] / pdf.value)
    # E[ybar(w) / pdf(w)] = integral of ybar = 1 after the observer's normalisation
    assert abs(np.mean(Ys) - 1.0) < 0.01
    w, wy = _tables.observer_y_weights()
    assert abs(wy.sum() - 1.0) < 1e-12


def test_oracle_white_furnace_cpu():
    scene, cam = scenes_render.white_furnace()
    tr = tracers.AdjointPhotonTracer()
    tr.maxRayGeneration = 2
    flat = R.flatten(scene)
    desc = R.render_desc(cam, 8, 8, 64, tr, seed=1)
    film = oracle.RenderScene(flat).render(desc)
    mean, var = R.resolve(film)
    centre = mean[3:5, 3:5, 1]
    assert np.all(np.abs(centre - 1.0) < 0.25), centre


def test_oracle_cornell_is_deterministic_and_lit():
    e = scenes_render.cornell_engine(16, 16, 4)
    flat = R.flatten(e.scene)
    desc = R.render_desc(e.camera, 16, 16, 4, e.tracer)
    a = oracle.RenderScene(flat).render(desc)
    b = oracle.RenderScene(flat).render(desc, threads=1)
    np.testing.assert_array_equal(a, b)
    assert R.resolve(a)[0][..., 1].mean() > 0.01
