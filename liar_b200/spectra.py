"""Spectra of the scene API: ``liar.spectra`` (src/liar/spectra/) plus the flat ``Spectrum``.

All wavelengths are in metres, like the reference. A spectrum is evaluated at one wavelength per
sample on the GPU (the reference's Spectral `Single` mode, src/liar/kernel/spectral.cpp:178-220);
here the classes only record their parameters, and :meth:`__call__` evaluates them on the host for
luminance and tests.
"""
from __future__ import annotations

import numpy as np

from . import _tables


class Spectrum:
    """Base of all spectra. ``Spectrum(value)`` is a flat spectrum."""

    def __init__(self, value: float = 1.0):
        self.value = float(value)

    def __call__(self, wavelength):
        return np.full(np.shape(wavelength), self.value, dtype=np.float64)

    @property
    def luminance(self) -> float:
        """Y of the spectrum under the standard observer (Spectrum::luminance, kernel/spectrum.cpp:93)."""
        w, weights = _tables.observer_y_weights()
        return float(np.sum(weights * self(w)))

    def isChromatic(self) -> bool:
        return False


class Sampled(Spectrum):
    """Piecewise linear spectrum through (wavelengths, values) (spectra/sampled.cpp)."""

    def __init__(self, wavelengths, values):
        self.wavelengths = tuple(float(w) for w in wavelengths)
        self.values = tuple(float(v) for v in values)
        if len(self.wavelengths) != len(self.values) or len(self.wavelengths) < 2:
            raise ValueError("Sampled needs as many values as wavelengths, at least two")
        if any(b <= a for a, b in zip(self.wavelengths, self.wavelengths[1:])):
            raise ValueError("wavelengths must be strictly increasing")

    def __call__(self, wavelength):
        # Sampled::doCall (spectra/sampled.cpp:104-126): zero outside the table
        w = np.asarray(wavelength, dtype=np.float64)
        ws = np.asarray(self.wavelengths)
        out = np.interp(w, ws, np.asarray(self.values))
        return np.where((w < ws[0]) | (w > ws[-1]), 0.0, out)

    def resample(self, wavelengths) -> "Sampled":
        """Sampled::resample (spectra/sampled.cpp:76-101): piecewise linear on [w0, wn), 0 elsewhere."""
        ws = [float(w) for w in wavelengths]
        out = [0.0] * len(ws)
        i, n = 0, len(ws)
        while i < n and ws[i] < self.wavelengths[0]:
            i += 1
        for k in range(1, len(self.wavelengths)):
            w1, w2 = self.wavelengths[k - 1], self.wavelengths[k]
            while i < n and ws[i] < w2:
                t = (ws[i] - w1) / (w2 - w1)
                out[i] = self.values[k - 1] + t * (self.values[k] - self.values[k - 1])
                i += 1
        return Sampled(ws, out) if len(ws) >= 2 else _Resampled(ws, out)

    def isChromatic(self) -> bool:
        return len(set(self.values)) > 1


class _Resampled(Spectrum):
    def __init__(self, ws, vs):
        self.wavelengths, self.values = tuple(ws), tuple(vs)


class BlackBody(Spectrum):
    """Planck's law normalised to 1 at its peak, times scale (spectra/black_body.cpp:44-118)."""

    def __init__(self, temperature: float, scale: float = 1.0):
        self.temperature = float(temperature)
        self.scale = float(scale)

    @property
    def peakWavelength(self) -> float:
        return 2.897771955e-3 / self.temperature

    @staticmethod
    def _planck(w, T):
        h, c, kb = 6.626070040e-34, 299792458.0, 1.3806488e-23
        return 2 * h * c * c / (w ** 5 * np.expm1(h * c / (kb * w * T)))

    def __call__(self, wavelength):
        w = np.asarray(wavelength, dtype=np.float64)
        return self.scale * self._planck(w, self.temperature) / self._planck(self.peakWavelength, self.temperature)

    def isChromatic(self) -> bool:
        return True


class Cauchy(Spectrum):
    """Refractive index a + b / lambda_um^2 (spectra/cauchy.cpp:72-80)."""

    def __init__(self, a: float, b: float = 0.0):
        self.a = float(a)
        self.b = float(b)

    def __call__(self, wavelength):
        w = np.asarray(wavelength, dtype=np.float64) * 1e6
        return self.a + self.b / (w * w)

    def isChromatic(self) -> bool:
        return self.b != 0.0


class Xyz(Spectrum):
    """A spectrum given by its tristimulus value (the reference's SpectrumXYZ,
    kernel/spectrum.cpp:232-252), evaluated through the standard recovery (liar_b200.recovery)."""

    def __init__(self, xyz):
        self.xyz = tuple(float(v) for v in xyz)
        if len(self.xyz) != 3:
            raise ValueError("Xyz needs three values")

    def __call__(self, wavelength):
        from .recovery import standard
        rec = standard()
        w = np.asarray(wavelength, dtype=np.float64)
        return np.vectorize(lambda x: rec.recover(self.xyz, x))(w).astype(np.float64)

    @property
    def luminance(self) -> float:
        return self.xyz[1]

    def isChromatic(self) -> bool:
        return True


def rgb(r, g=None, b=None, space=None) -> Xyz:
    """rgb(r, g, b[, space]) or rgb((r, g, b)[, space]) (kernel/rgb_space.cpp:402-419): the colour in
    the RGB space (sRGB by default) as a tristimulus spectrum."""
    from .recovery import sRGB, RgbSpace
    if g is None or isinstance(g, RgbSpace):
        space = g if isinstance(g, RgbSpace) else space
        r, g, b = tuple(r)[:3]
    return Xyz((space or sRGB).toXYZ((r, g, b)))


def spd(name: str, component: str = "n") -> Sampled:
    """Complex refractive index table of a metal (Ag, Al, Au, Cu) as a Sampled spectrum of n or k,
    the data the reference ships as data/spd/*.spd (read by src/liar/tools/spd.py)."""
    rows = _tables.spd(name)
    col = {"n": 1, "k": 2}[component]
    return Sampled([r[0] for r in rows], [r[col] for r in rows])
