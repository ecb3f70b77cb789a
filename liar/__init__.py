"""``liar``: the reference's package name over liar_b200, so that a LiAR scene script runs unchanged.

A script starts with ``from liar import *`` and ``from liar.tools import cornell_box, scripting``
(the reference's package layout, src/liar/__init__.py:37-79). This package registers liar_b200's
modules under the reference's names (``liar.scenery``, ``liar.shaders``, ``liar.kernel`` ...),
exports the same top-level names, and holds the ``liar.tools`` helpers. Everything renders through
liar_b200 on the GPU; there is no CPU fallback. The standard observer and the Meng-Simon recovery
that the reference loads at import (``Observer.setStandard``, ``Recovery.setStandard``) are
liar_b200's built-in tables.
"""
from __future__ import annotations

import sys as _sys

import liar_b200 as _impl
from liar_b200 import (cameras, kernel, mediums, output, samplers, scenery, shaders,  # noqa: F401
                       spectra, textures, tracers)
from liar_b200 import codecs  # noqa: F401
from liar_b200.kernel import RenderEngine, setTolerance, tolerance  # noqa: F401
from liar_b200.recovery import CIEXYZ, RgbSpace, sRGB  # noqa: F401
from liar_b200.spectra import rgb  # noqa: F401

for _name in ("cameras", "codecs", "kernel", "mediums", "output", "samplers", "scenery", "shaders", "spectra",
              "textures", "tracers"):
    _sys.modules[f"{__name__}.{_name}"] = getattr(_impl, _name)

# the kernel's names (from liar.kernel import *, src/liar/kernel/kernel_init.cpp:82-160)
kernel.RenderEngine = RenderEngine
kernel.rgb = rgb
kernel.RgbSpace = RgbSpace
kernel.sRGB = sRGB
kernel.CIEXYZ = CIEXYZ

__all__ = ["cameras", "codecs", "kernel", "mediums", "output", "samplers", "scenery", "shaders", "spectra",
           "textures", "tracers", "RenderEngine", "rgb", "RgbSpace", "sRGB", "CIEXYZ", "tolerance", "setTolerance"]
