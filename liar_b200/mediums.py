"""Participating media of the scene API (``liar.mediums``, src/liar/mediums/).

The classes keep their parameters so that a scene script builds unchanged, but media are not on
the GPU path: rendering a scene in which an object's ``interior`` (or the engine's) is a medium
other than Vacuum raises NotImplementedError.
"""
from __future__ import annotations


class Medium:
    def __init__(self):
        self.priority = 0


class Vacuum(Medium):
    """The empty medium (the reference's default interior)."""


class Beer(Medium):
    """Beer(transparency): Beer-Lambert absorption (mediums/beer.cpp)."""

    def __init__(self, transparency=None):
        super().__init__()
        self.transparency = transparency


class Fog(Medium):
    """Fog([extinction[, assymetry]]) (mediums/fog.cpp)."""

    def __init__(self, extinction=None, assymetry: float = 0.0):
        super().__init__()
        self.extinction = extinction
        self.assymetry = float(assymetry)
        self.color = None
        self.emission = None
        self.numScatterSamples = 1


class ExponentialFog(Fog):
    """ExponentialFog (mediums/exponential_fog.cpp)."""

    def __init__(self, extinction=None, assymetry: float = 0.0):
        super().__init__(extinction, assymetry)
        self.origin = (0.0, 0.0, 0.0)
        self.up = (0.0, 0.0, 1.0)
        self.decay = 1.0


class Bounded(Medium):
    """Bounded(medium, bounds) (mediums/bounded.cpp)."""

    def __init__(self, medium=None, bounds=None):
        super().__init__()
        self.medium = medium
        self.bounds = bounds


def is_vacuum(medium) -> bool:
    return medium is None or isinstance(medium, Vacuum)
