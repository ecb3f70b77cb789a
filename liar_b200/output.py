"""Render targets (``liar.output``). Image keeps the reference's name and writes its file through
the reference's Raster tone mapping (output/raster.cpp) and image codecs (``codecs.py``: .png,
.hdr, .pfm, .exr); a name ending in .npy keeps the linear XYZA film itself. Display, an X11
window in the reference, is unavailable on this box and is replaced by a headless buffer that
keeps the last frame."""
from __future__ import annotations

import enum
import math
from pathlib import Path

import numpy as np

from . import codecs

TONE_MAPPINGS = ("Linear", "CompressY", "CompressRGB", "Reinhard2002Y", "Reinhard2002RGB", "ExponentialY",
                 "ExponentialRGB", "DuikerY", "DuikerRGB")


class ToneMapping(str, enum.Enum):
    """Raster.ToneMapping, a string enum as in the reference (output/raster.cpp:29-41)."""

    Linear = "Linear"
    CompressY = "CompressY"
    CompressRGB = "CompressRGB"
    Reinhard2002Y = "Reinhard2002Y"
    Reinhard2002RGB = "Reinhard2002RGB"
    ExponentialY = "ExponentialY"
    ExponentialRGB = "ExponentialRGB"
    DuikerY = "DuikerY"
    DuikerRGB = "DuikerRGB"


def _filmic(x):
    """Duiker's filmic curve with the display gamma undone (raster.cpp:60-67)."""
    x = np.maximum(np.float32(0), x - np.float32(0.004))
    y = (x * (np.float32(6.2) * x + np.float32(0.5))) / (x * (np.float32(6.2) * x + np.float32(1.7)) + np.float32(0.06))
    return np.power(y, np.float32(2.2))


def _inv_filmic(y: float) -> float:
    y = min(max(y, 0.0), 0.99999) ** (1.0 / 2.2)
    a, b, c = 6.2 * y - 6.2, 1.7 * y - 0.5, 0.06 * y
    return (-b - math.sqrt(b * b - 4 * a * c)) / (2 * a) + 0.004


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

    def isCanceling(self) -> bool:
        """RenderTarget::isCanceling (kernel/render_target.h:59): True asks the engine to stop the
        render in progress. The base target never cancels; a subclass may override it."""
        return False


class Raster(RenderTarget):
    """The reference's Raster settings and tone mapping (output/raster.cpp:45-500): rgbSpace,
    toneMapping, exposureStops (setting it turns autoExposure off), exposureCorrectionStops,
    autoExposure (default on), middleGrey (0.184)."""

    def __init__(self, resolution=(320, 240)):
        super().__init__(resolution)
        self.rgbSpace = codecs.default_space()
        self._tone = "Linear"
        self._stops = 0.0
        self.exposureCorrectionStops = 0.0
        self.autoExposure = True
        self.middleGrey = 0.184

    @property
    def toneMapping(self) -> str:
        return self._tone

    ToneMapping = ToneMapping

    @toneMapping.setter
    def toneMapping(self, mode: str):
        name = str(getattr(mode, "value", mode))
        for t in TONE_MAPPINGS:
            if t.lower() == name.lower():
                self._tone = t
                return
        raise KeyError(f"unknown tone mapping {mode!r}; one of {TONE_MAPPINGS}")

    @property
    def exposureStops(self) -> float:
        if self.autoExposure and self.xyza is not None:
            return self._auto_stops()
        return self._stops

    @exposureStops.setter
    def exposureStops(self, stops: float):
        self.autoExposure = False
        self._stops = float(stops)

    def _auto_stops(self) -> float:
        """Raster::exposureStops with autoExposure (raster.cpp:99-150): the gain that maps the
        log-average luminance of the covered pixels to middleGrey, in thirds of a stop."""
        y = self.xyza[..., 1].astype(np.float64)
        cov = y > 0
        if not cov.any():
            gain = 1.0
        else:
            avg = math.exp(float(np.log(y[cov]).mean()))
            g = self.middleGrey
            if self._tone == "Linear":
                gain = g / avg
            elif self._tone in ("CompressY", "CompressRGB", "Reinhard2002Y", "Reinhard2002RGB"):
                gain = g / (avg * (1 - g))
            elif self._tone in ("ExponentialY", "ExponentialRGB"):
                gain = -math.log1p(-g) / avg
            else:
                gain = _inv_filmic(g) / avg
        self._stops = round(3.0 * math.log2(gain)) / 3.0
        return self._stops

    def tonemap(self, space) -> np.ndarray:
        """Raster::tonemap(destSpace) (raster.cpp:309-496): (H, W, 4) RGBA in `space`; a NaN
        pixel becomes pink."""
        gain = np.float32(2.0 ** (self.exposureStops + self.exposureCorrectionStops))
        lin = self.xyza[..., :3].astype(np.float32) * gain
        alpha = self.xyza[..., 3:4].astype(np.float32)
        t = self._tone
        with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
            if t == "Linear":
                rgb = space.toRGB(lin)
            elif t == "CompressY":
                rgb = space.toRGB(lin / (1 + lin[..., 1:2]))
            elif t == "ExponentialY":
                Y = lin[..., 1:2]
                scale = np.where(Y < 1e-8, 1 - Y / 2, -np.expm1(-Y) / Y)
                rgb = space.toRGB(lin * scale)
            elif t == "DuikerY":
                Y = lin[..., 1:2]
                rgb = space.toRGB(lin * (_filmic(Y) / np.maximum(Y, np.float32(0.004))))
            elif t == "Reinhard2002Y":
                Lw = gain * np.float32(self.max_scene_luminance())
                inv = np.float32(1.0) / (Lw * Lw)
                Y = lin[..., 1:2]
                rgb = space.toRGB(lin * ((1 + Y * inv) / (1 + Y)))
            else:
                c = space.toRGBlinear(lin)
                if t == "CompressRGB":
                    c = c / (1 + c)
                elif t == "Reinhard2002RGB":
                    Lw = gain * np.float32(self.max_scene_luminance())
                    inv = np.float32(1.0) / (Lw * Lw)
                    c = c * (1 + c * inv) / (1 + c)
                elif t == "ExponentialRGB":
                    c = -np.expm1(-c)
                else:  # DuikerRGB
                    c = _filmic(c)
                rgb = space.toGamma(c)
        out = np.concatenate([rgb, alpha], axis=-1).astype(np.float32)
        bad = np.isnan(out).any(axis=-1)
        out[bad] = (1.0, 0.0, 1.0, 1.0)
        return out

    def max_scene_luminance(self) -> float:
        """The brightest pixel's mean luminance (the reference tracks it while splatting,
        raster.cpp:594-598)."""
        y = self.xyza[..., 1]
        return float(max(y.max(), 0.0)) if y.size else 0.0


class Image(Raster):
    """Image(path, resolution) (output/image.cpp): on writing, the film tone-mapped into the codec's
    colour space and saved (Image::save); a .npy path keeps the linear XYZA film."""

    def __init__(self, path: str = "image.npy", resolution=(320, 240)):
        super().__init__(resolution)
        self.path = path
        self.options = ""

    @property
    def filename(self) -> str:
        return str(self.path)

    @filename.setter
    def filename(self, value: str):
        self.path = value

    def write(self, xyza, variance):
        super().write(xyza, variance)
        self.save()

    def save(self):
        p = Path(self.path)
        if p.suffix.lower() == ".npy":
            np.save(p, self.xyza.astype(np.float32))
            return
        space = codecs.writer_space(p, self.rgbSpace)
        codecs.write(p, self.tonemap(space), space)


class Display(Raster):
    """Display(title, resolution): the reference's window (output/display.cpp, PixelToaster) is
    unavailable on this box; this headless raster keeps the last frame (``xyza``, and
    ``tonemap(space)`` for its pixels) with the window's settings."""

    def __init__(self, title: str = "", resolution=(320, 240)):
        super().__init__(resolution)
        self._title = str(title)
        self.autoUpdate = True
        self.showHistogram = False

    @property
    def title(self) -> str:
        return self._title


class Splitter(RenderTarget):
    """Splitter([children]) (output/splitter.cpp): hands every render to each child; its resolution
    is the children's largest; it is cancelling when any child is."""

    def __init__(self, children=()):
        self.children = list(children)
        super().__init__(self.resolution)

    @property
    def resolution(self) -> tuple[int, int]:
        w, h = 1, 1
        for c in getattr(self, "_children", []):
            w, h = max(w, c.resolution[0]), max(h, c.resolution[1])
        return (w, h)

    @resolution.setter
    def resolution(self, value) -> None:  # derived from the children
        pass

    @property
    def children(self) -> list:
        return list(self._children)

    @children.setter
    def children(self, children) -> None:
        self._children = list(children)

    def add(self, child) -> None:
        if isinstance(child, (list, tuple)):
            self._children.extend(child)
        else:
            self._children.append(child)

    def write(self, xyza, variance):
        super().write(xyza, variance)
        for c in self._children:
            c.write(xyza, variance)

    def isCanceling(self) -> bool:
        return any(c.isCanceling() for c in self._children)


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
    maxSampleLuminance of the raster at the end of the chain. A Splitter's children share the one
    GPU film, so they must agree on these settings."""
    if isinstance(target, Splitter):
        settings = [film_settings(c) for c in target.children] or [film_settings(None)]
        if any(st != settings[0] for st in settings[1:]):
            raise NotImplementedError("the children of a Splitter render into one film: give them the same filter "
                                      "and maxSampleLuminance")
        return settings[0]
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
