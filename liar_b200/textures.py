"""Textures of the scene API (``liar.textures``). Only constant textures are on the hot path
(src/liar/textures/constant.cpp); a Constant wraps a spectrum or a number."""
from __future__ import annotations

from .spectra import Spectrum


class Texture:
    pass


class Constant(Texture):
    def __init__(self, value=1.0):
        self.value = value if isinstance(value, Spectrum) else Spectrum(float(value))

    @property
    def spectrum(self) -> Spectrum:
        return self.value


def as_spectrum(x) -> Spectrum:
    """Spectrum of a texture, a spectrum or a number (the shaders' texture slots)."""
    if isinstance(x, Constant):
        return x.value
    if isinstance(x, Spectrum):
        return x
    if isinstance(x, (int, float)):
        return Spectrum(float(x))
    raise TypeError(f"unsupported texture {type(x).__name__}: only constant textures are implemented")


def as_scalar(x) -> float:
    """Scalar of a texture slot that the shaders read with scalarLookUp (roughness)."""
    s = as_spectrum(x)
    if type(s) is Spectrum:
        return s.value
    raise TypeError("roughness textures must be flat")
