"""liar_b200 -- B200 (sm_100a) implementation of LiAR's per-sample rendering hot path.

The package mirrors the reference's Python scene API (``from liar import *``): the sub-modules
``scenery``, ``shaders``, ``spectra``, ``textures``, ``cameras``, ``samplers``, ``tracers``,
``output`` and ``RenderEngine``. The scene objects only record parameters; the traversal,
shading and photon work runs on the GPU behind the C ABI of include/liar_gpu.h
(``libliar_gpu.so``, built by ``python -m liar_b200.build``). There is no CPU fallback.
"""
from . import cameras, mediums, output, samplers, scenery, shaders, spectra, textures, tracers  # noqa: F401
from .kernel import RenderEngine, setTolerance, tolerance  # noqa: F401
from .recovery import CIEXYZ, RgbSpace, sRGB  # noqa: F401
from .spectra import rgb  # noqa: F401

__all__ = ["cameras", "mediums", "output", "samplers", "scenery", "shaders", "spectra", "textures", "tracers",
           "RenderEngine", "rgb", "RgbSpace", "sRGB", "CIEXYZ", "tolerance", "setTolerance"]
