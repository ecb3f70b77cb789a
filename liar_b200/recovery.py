"""Spectra from tristimulus values: the reference's standard recovery, RecoveryMengSimon
(src/liar/spectra/recovery_meng_simon.cpp:93-310, loaded as the standard one by
src/liar/__init__.py:72-79), after Meng, Simon, Hanika and Dachsbacher, "Physically Meaningful
Rendering using Tristimulus Colours" (EGSR 2015).

The table holds spectra sampled at a set of chromaticities xy. Those points and the four corners
of the box [-0.3, 1.0] x [-0.3, 1.2] are triangulated (Delaunay, which is what the reference's
planar mesh maintains while it inserts the sites); a colour XYZ whose chromaticity lies in the
box is the barycentric blend of the spectra at the corners of the triangle that contains it, the
box corners carrying the zero spectrum, with the weights scaled to sum to X + Y + Z
(RecoveryMengSimon::Impl::recover). At a wavelength the blend is interpolated linearly between
the table's wavelengths and is zero outside them; as a reflectance it is divided by the blend of
the spectra's maxima when that exceeds 1 (doRecover, Single mode).

Also the reference's RGB colours: ``rgb(r, g, b)`` (kernel/rgb_space.cpp:402-419) converts with
the default RGB space, sRGB with gamma 2.2 and Bradford adaptation from its white point to
illuminant E (kernel/rgb_space.h:135-140, rgb_space.cpp:315-380, 424-444), and makes a spectrum
of the XYZ value, recovered as above.
"""
from __future__ import annotations

import functools

import numpy as np

from . import _tables

BOX_LO = (-0.3, -0.3)
BOX_HI = (1.0, 1.2)


class RecoveryMengSimon:
    """RecoveryMengSimon(wavelengths, {(x, y): values}) with wavelengths in metres."""

    def __init__(self, wavelengths, samples):
        from scipy.spatial import Delaunay

        self.wavelengths = np.asarray(wavelengths, dtype=np.float32)
        if self.wavelengths.size < 2 or np.any(np.diff(self.wavelengths) <= 0):
            raise ValueError("RecoveryMengSimon needs at least two strictly increasing wavelengths")
        items = list(samples.items()) if isinstance(samples, dict) else list(samples)
        xy = np.asarray([k for k, _ in items], dtype=np.float64)
        vals = np.asarray([v for _, v in items], dtype=np.float32)
        if vals.shape != (len(items), self.wavelengths.size):
            raise ValueError("RecoveryMengSimon needs as many values as wavelengths per sample")
        if np.any(xy < BOX_LO) or np.any(xy > BOX_HI):
            raise ValueError("chromaticities must lie in the box [-0.3, 1.0] x [-0.3, 1.2]")
        corners = np.array([[BOX_LO[0], BOX_LO[1]], [BOX_HI[0], BOX_LO[1]], [BOX_HI[0], BOX_HI[1]],
                            [BOX_LO[0], BOX_HI[1]]])
        self.n_samples = len(items)
        self.points = np.concatenate([xy, corners])
        self.values = vals                       # (n_samples, n_wavelengths)
        self.maxima = vals.max(axis=1)           # PointInfo::max
        self.triangulation = Delaunay(self.points)

    def locate(self, xyz) -> tuple[np.ndarray, np.ndarray] | None:
        """(sample indices (-1 for a box corner), weights) of the blend for XYZ, or None when the
        colour has no recovery (zero sum or chromaticity outside the box)."""
        X, Y, Z = (np.float32(v) for v in xyz)
        s = np.float32(X + Y + Z)
        if s == 0:
            return None
        x, y = np.float32(X / s), np.float32(Y / s)
        if not (BOX_LO[0] <= x <= BOX_HI[0] and BOX_LO[1] <= y <= BOX_HI[1]):
            return None
        tri = int(self.triangulation.find_simplex(np.array([[x, y]], dtype=np.float64))[0])
        if tri < 0:
            return None
        verts = self.triangulation.simplices[tri]
        T = self.triangulation.transform[tri]
        b = T[:2] @ (np.array([x, y], dtype=np.float64) - T[2])
        w = np.array([b[0], b[1], 1.0 - b[0] - b[1]], dtype=np.float32)
        idx = np.where(verts < self.n_samples, verts, -1)
        w[idx < 0] = 0.0
        wtot = np.float32(w.sum())
        if wtot == 0:
            return None
        w = (w * np.float32(s / wtot)).astype(np.float32)
        return idx, w

    def sampled(self, xyz) -> tuple[np.ndarray, np.ndarray, float]:
        """The blended spectrum at the table's wavelengths and the blend of the maxima."""
        loc = self.locate(xyz)
        n = self.wavelengths.size
        if loc is None:
            return self.wavelengths.copy(), np.zeros(n, np.float32), 0.0
        idx, w = loc
        acc = np.zeros(n, np.float32)
        mx = np.float32(0.0)
        for i, wi in zip(idx, w):
            if i >= 0:
                acc = (acc + wi * self.values[i]).astype(np.float32)
                mx = np.float32(mx + wi * self.maxima[i])
        return self.wavelengths.copy(), acc, float(mx)

    def recover(self, xyz, wavelength: float, reflectant: bool = False) -> float:
        ws, vs, mx = self.sampled(xyz)
        k = int(np.searchsorted(ws, np.float32(wavelength), side="right"))
        if k == 0 or k == ws.size:
            return 0.0
        t = (np.float32(wavelength) - ws[k - 1]) / (ws[k] - ws[k - 1])
        v = float(vs[k - 1] + t * (vs[k] - vs[k - 1]))
        if reflectant and mx > 1.0:
            return v / mx
        return v


@functools.lru_cache(maxsize=None)
def standard() -> RecoveryMengSimon:
    """The standard recovery of the reference (its data/recovery_meng_simon.json table)."""
    t = _tables.recovery()
    return RecoveryMengSimon(t["wavelengths"], [(tuple(xy), v) for xy, v in zip(t["xy"], t["spectra"])])


def device_table(rec: RecoveryMengSimon | None = None) -> dict:
    """The arrays liar_gpu_set_recovery takes: wavelengths, xy, spectra and the triangles (point
    indices; the box corners follow the samples)."""
    rec = rec or standard()
    return {"wavelengths": np.ascontiguousarray(rec.wavelengths, dtype=np.float32),
            "xy": np.ascontiguousarray(rec.points[:rec.n_samples], dtype=np.float32),
            "points": np.ascontiguousarray(rec.points, dtype=np.float32),
            "spectra": np.ascontiguousarray(rec.values, dtype=np.float32),
            "triangles": np.ascontiguousarray(rec.triangulation.simplices, dtype=np.int32)}


def set_standard_on(ctx) -> None:
    """Sets the standard recovery on a device context (once per context)."""
    import ctypes as C
    if getattr(ctx, "_recovery_set", False):
        return
    t = device_table()
    fn = ctx._lib.liar_gpu_set_recovery
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int]
    ctx.check(fn(ctx.handle, t["wavelengths"].ctypes.data, t["wavelengths"].size, t["xy"].ctypes.data,
                 t["spectra"].ctypes.data, t["xy"].shape[0], t["triangles"].ctypes.data, t["triangles"].shape[0]))
    ctx._recovery_set = True


# ---- RGB spaces (kernel/rgb_space.cpp)

_BRADFORD = np.array([[0.8951, 0.2664, -0.1614], [-0.7502, 1.7135, 0.0367], [0.0389, -0.0685, 1.0296]])


class RgbSpace:
    """RgbSpace(red, green, blue, white, gamma): chromaticities of the primaries and the white point."""

    def __init__(self, red, green, blue, white, gamma: float = 1.0):
        for c in (red, green, blue, white):
            if c[0] < 0 or c[1] < 0 or c[0] + c[1] > 1.001:
                raise ValueError(f"invalid chromaticity {c}")
        if white[1] == 0 or gamma <= 0:
            raise ValueError("bad white point or gamma")
        self.red, self.green, self.blue, self.white, self.gamma = red, green, blue, white, float(gamma)
        prim = np.array([[red[0], green[0], blue[0]], [red[1], green[1], blue[1]],
                         [1 - red[0] - red[1], 1 - green[0] - green[1], 1 - blue[0] - blue[1]]])
        W = np.array([white[0] / white[1], 1.0, (1 - white[0] - white[1]) / white[1]])
        S = np.linalg.solve(prim, W)
        m_xyz = prim * S[None, :]                      # linear RGB -> XYZ (white W)
        cs, cd = _BRADFORD @ W, _BRADFORD @ np.ones(3)
        m_cat = np.linalg.inv(_BRADFORD) @ np.diag(cd / cs) @ _BRADFORD   # white W -> illuminant E
        self.matrix = (m_cat @ m_xyz).astype(np.float32)  # columns: XYZ of the red, green, blue primaries
        self.inverse = np.linalg.inv(m_cat @ m_xyz).astype(np.float32)  # columns: RGB of X, Y, Z

    def toXYZ(self, rgb) -> tuple[float, float, float]:
        r = np.asarray(rgb[:3], dtype=np.float32)
        if self.gamma != 1.0:
            r = (np.sign(r) * np.power(np.abs(r), np.float32(self.gamma))).astype(np.float32)  # tonecurve
        x = self.matrix[:, 0] * r[0] + self.matrix[:, 1] * r[1] + self.matrix[:, 2] * r[2]
        return tuple(float(v) for v in x.astype(np.float32))

    # array forms (..., 3) of RgbSpace::toXYZ / toRGBA / toRGBAlinear / toGamma / toLinear
    # (rgb_space.cpp:82-189); the tonecurve is sign(x) |x|^gamma
    def _curve(self, a: np.ndarray, g: float) -> np.ndarray:
        if g == 1.0:
            return a
        return (np.sign(a) * np.power(np.abs(a), np.float32(g))).astype(np.float32)

    def toLinear(self, rgb) -> np.ndarray:
        return self._curve(np.asarray(rgb, dtype=np.float32), self.gamma)

    def toGamma(self, rgb) -> np.ndarray:
        return self._curve(np.asarray(rgb, dtype=np.float32), 1.0 / self.gamma)

    def toXYZlinear(self, rgb) -> np.ndarray:
        return (np.asarray(rgb, dtype=np.float32) @ self.matrix.T).astype(np.float32)

    def toXYZarray(self, rgb) -> np.ndarray:
        return self.toXYZlinear(self.toLinear(rgb))

    def toRGBlinear(self, xyz) -> np.ndarray:
        return (np.asarray(xyz, dtype=np.float32) @ self.inverse.T).astype(np.float32)

    def toRGB(self, xyz) -> np.ndarray:
        return self.toGamma(self.toRGBlinear(xyz))

    def withGamma(self, gamma: float) -> "RgbSpace":
        return RgbSpace(self.red, self.green, self.blue, self.white, gamma)

    def linearSpace(self) -> "RgbSpace":
        return self.withGamma(1.0)

    def __eq__(self, other) -> bool:
        return isinstance(other, RgbSpace) and (self.red, self.green, self.blue, self.white, self.gamma) == \
            (other.red, other.green, other.blue, other.white, other.gamma)

    def __hash__(self) -> int:
        return hash((self.red, self.green, self.blue, self.white, self.gamma))


sRGB = RgbSpace((0.6400, 0.3300), (0.3000, 0.6000), (0.1500, 0.0600), (0.3127, 0.3290), 2.2)
# the identity space of the reference (kernel/rgb_space.h:126-130): X, Y, Z as R, G, B, white E
CIEXYZ = RgbSpace((1.0, 0.0), (0.0, 1.0), (0.0, 0.0), (1.0 / 3, 1.0 / 3), 1.0)
