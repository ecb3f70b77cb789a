"""Render targets (``liar.output``). Image keeps the reference's name; with no image codecs in this
build it writes the linear XYZ film as .npy (or a 3-channel .pfm when the name ends in .pfm).
Display, an X11 window in the reference, is unavailable on this box and is replaced by a headless
buffer that keeps the last frame."""
from __future__ import annotations

from pathlib import Path

import numpy as np


class RenderTarget:
    def __init__(self, resolution=(320, 240)):
        self.resolution = (int(resolution[0]), int(resolution[1]))
        self.xyza = None      # (H, W, 4) mean X, Y, Z, alpha
        self.variance = None  # (H, W, 3) variance of the per-pixel mean of X, Y, Z

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
