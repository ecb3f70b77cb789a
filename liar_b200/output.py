"""Render targets (``liar.output``). Image keeps the reference's name; with no image codecs in this
build it writes the linear XYZ film as .npy (or a 3-channel .pfm when the name ends in .pfm).
Display, an X11 window in the reference, is unavailable on this box and is replaced by a headless
buffer that keeps the last frame."""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np


class RenderTarget:
    def __init__(self, resolution=(320, 240)):
        self.resolution = (int(resolution[0]), int(resolution[1]))
        self.xyza = None      # (H, W, 4) mean X, Y, Z, alpha
        self.variance = None  # (H, W, 3) variance of the per-pixel mean of X, Y, Z
        # Raster.maxSampleLuminance (output/raster.cpp:572-575): samples brighter in Y are scaled
        # down to it; infinity (the reference's default) keeps them
        self.maxSampleLuminance = math.inf

    def write(self, xyza: np.ndarray, variance: np.ndarray) -> None:
        self.xyza = xyza
        self.variance = variance


class Image(RenderTarget):
    def __init__(self, filename: str = "image.npy", resolution=(320, 240)):
        super().__init__(resolution)
        self.filename = filename

    def write(self, xyza, variance):
        super().write(xyza, variance)
        p = Path(self.filename)
        if p.suffix.lower() == ".pfm":
            h, w = xyza.shape[:2]
            with open(p, "wb") as f:
                f.write(f"PF\n{w} {h}\n-1.0\n".encode())
                f.write(np.ascontiguousarray(xyza[::-1, :, :3], dtype="<f4").tobytes())
        else:
            np.save(p.with_suffix(".npy") if p.suffix != ".npy" else p, xyza.astype(np.float32))


class Display(RenderTarget):
    def __init__(self, title: str = "", resolution=(320, 240)):
        super().__init__(resolution)
        self.title = title


class FilterTriangle(RenderTarget):
    """FilterTriangle(target[, width]) (output/filter_triangle.cpp): spreads every sample over the
    pixels within ceil(width) with weights max(0, width - |d|) per axis. Rendering through it
    selects the GPU film's triangle filter."""

    kind = 1

    def __init__(self, target, width: float = 1.0):
        super().__init__(target.resolution)
        self.target = target
        self.width = width

    @property
    def width(self) -> float:
        return self._width

    @width.setter
    def width(self, w: float) -> None:
        self._width = max(0.0, float(w))

    @property
    def filter_param(self) -> float:
        return self._width

    def write(self, xyza, variance):
        super().write(xyza, variance)
        self.target.write(xyza, variance)


class FilterMitchell(RenderTarget):
    """FilterMitchell(target[, b]) (output/filter_mitchell.cpp): the Mitchell-Netravali filter of
    radius 2 pixels with C = (1 - B) / 2, B = 1/3 by default."""

    kind = 2

    def __init__(self, target, b: float = 1.0 / 3.0):
        super().__init__(target.resolution)
        self.target = target
        self.b = float(b)

    @property
    def filter_param(self) -> float:
        return self.b

    def write(self, xyza, variance):
        super().write(xyza, variance)
        self.target.write(xyza, variance)


def film_settings(target) -> dict:
    """The GPU film settings of a render target chain: the outermost reconstruction filter and the
    maxSampleLuminance of the raster at the end of the chain."""
    filt, param = 0, 0.0
    t = target
    while isinstance(t, (FilterTriangle, FilterMitchell)):
        if filt == 0:
            filt, param = t.kind, t.filter_param
        t = t.target
    lum = getattr(t, "maxSampleLuminance", math.inf) if t is not None else math.inf
    if filt == 1 and param <= 0.0:
        raise ValueError("a triangle filter of width 0 gives no pixel any weight")
    return {"filter": filt, "filter_param": param, "max_sample_luminance": lum if math.isfinite(lum) else 0.0}
