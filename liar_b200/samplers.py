"""Samplers of the scene API (``liar.samplers``). Stratifier(resolution, samplesPerPixel) selects
the renderer's per-pixel stratified sampler (liar_b200/csrc/sampler.h), the counterpart of
src/liar/samplers/stratifier.cpp."""
from __future__ import annotations


class Stratifier:
    def __init__(self, resolution=(320, 240), samplesPerPixel: int = 1, jittered: bool = True):
        self.resolution = (int(resolution[0]), int(resolution[1]))
        self.samplesPerPixel = int(samplesPerPixel)
        self.jittered = jittered
        self.seed_ = 0

    def seed(self, value: int) -> None:
        self.seed_ = int(value)


class LatinHypercube(Stratifier):
    pass


class Halton(Stratifier):
    pass
