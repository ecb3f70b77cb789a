"""Samplers of the scene API (``liar.samplers``).

The renderer draws every sample value from a per-pixel hash sampler (liar_b200/csrc/sampler.h):
each dimension of a pixel is stratified over the pixel's samples, so any GPU thread can draw any
sample. The classes below select the reference's stratification patterns through the render
description's ``sampler`` bits:

* ``Stratifier`` (src/liar/samplers/stratifier.cpp): the samples per pixel are rounded to a
  square, as the reference does (``doSetSamplesPerPixel``, with its warning); screen and lens
  samples lie on the sqrt(spp) x sqrt(spp) grid of 2D strata (``doSampleScreen``, ``doSampleLens``).
* ``LatinHypercube`` (src/liar/samplers/latin_hypercube.cpp): any sample count; the screen and lens
  axes are stratified one by one over the samples, like every other dimension.
* ``jittered`` (both): False puts every stratified value at its stratum's centre (the reference's
  ``jitter()`` returns 0.5, samplers/stratifier.h:90).
* ``Halton`` (src/liar/samplers/halton.cpp) is a progressive sampler of the whole film (scrambled
  radical inverses of a global sample index, tasks of ``samplesPerTask`` samples); that render
  mode is not on the GPU path, and RenderEngine.render refuses it.
"""
from __future__ import annotations

import math

LIAR_SAMPLER_STRATIFIER = 0
LIAR_SAMPLER_LATIN_HYPERCUBE = 1
LIAR_SAMPLER_NOT_JITTERED = 2


class Sampler:
    def __init__(self):
        self.seed_ = 0

    def seed(self, value: int) -> None:
        self.seed_ = int(value)


class _Tiled(Sampler):
    _kind = LIAR_SAMPLER_STRATIFIER

    def __init__(self, resolution=(320, 240), samplesPerPixel: int = 1):
        super().__init__()
        self.resolution = resolution
        self.samplesPerPixel = samplesPerPixel
        self.jittered = True

    @property
    def resolution(self) -> tuple[int, int]:
        return self._resolution

    @resolution.setter
    def resolution(self, value) -> None:
        w, h = int(value[0]), int(value[1])
        if w <= 0 or h <= 0:
            raise ValueError(f"resolution must be positive, got {value!r}")
        self._resolution = (w, h)

    @property
    def samplesPerPixel(self) -> int:
        return self._spp

    @samplesPerPixel.setter
    def samplesPerPixel(self, value: int) -> None:
        self._spp = max(int(value), 1)

    @property
    def jittered(self) -> bool:
        return self._jittered

    @jittered.setter
    def jittered(self, value: bool) -> None:
        self._jittered = bool(value)

    @property
    def mode(self) -> int:
        """The render description's LIAR_SAMPLER_* bits."""
        return self._kind | (0 if self._jittered else LIAR_SAMPLER_NOT_JITTERED)


class Stratifier(_Tiled):
    """Stratifier([resolution[, samplesPerPixel]]): jittered stratified sampling; the sample count
    is rounded to the nearest square (stratifier.cpp doSetSamplesPerPixel)."""

    _kind = LIAR_SAMPLER_STRATIFIER

    @_Tiled.samplesPerPixel.setter
    def samplesPerPixel(self, value: int) -> None:
        n = int(value)
        axis = max(int(round(math.sqrt(max(n, 1)))), 1)
        if axis * axis != n:
            print(f"Sampler warning: samples per pixel: using size {axis * axis} instead of {n}")
        self._spp = axis * axis


class LatinHypercube(_Tiled):
    """LatinHypercube([resolution[, samplesPerPixel]]): every axis stratified on its own."""

    _kind = LIAR_SAMPLER_LATIN_HYPERCUBE


class Halton(Sampler):
    """Halton(): the reference's progressive scrambled-Halton sampler. Its parameters are kept, but
    rendering with it raises NotImplementedError: progressive film-wide sampling is not on the GPU
    path (use Stratifier or LatinHypercube)."""

    progressive = True

    def __init__(self):
        super().__init__()
        self.samplesPerTask = 1024
