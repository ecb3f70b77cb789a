"""Saving and loading a flattened scene and its render description (test fixtures).

A fixture is one .npz file: the FlatScene's arrays as they are, its ctypes record arrays
(materials, spectra, lights, textures) as raw bytes with their counts, and the CRenderDesc as raw
bytes. Loading rebuilds the same FlatScene and CRenderDesc, so that a GPU test can render exactly
what a scene script asked for."""
from __future__ import annotations

import ctypes as C

import numpy as np

from liar_b200 import render as R

_ARRAYS = ("vertices", "triangles", "triangle_object", "normals", "triangle_normals", "object_material",
           "object_light", "pool", "observer", "triangle_uvs", "texture_pixels", "noise_tables", "spheres",
           "sphere_object")
_RECORDS = {"materials": R.CMaterial, "spectra": R.CSpectrum, "lights": R.CLight, "textures": R.CTexture}


def save(path, flat: R.FlatScene, desc: R.CRenderDesc, **extra) -> None:
    out = {}
    for k in _ARRAYS:
        v = getattr(flat, k)
        if v is not None:
            out["a_" + k] = np.asarray(v)
    for k in _RECORDS:
        v = getattr(flat, k)
        if v is not None:
            out["r_" + k] = np.frombuffer(bytes(v), dtype=np.uint8)
            out["n_" + k] = np.int64(len(v))
    out["scene_radius"] = np.float32(flat.scene_radius)
    out["desc"] = np.frombuffer(bytes(desc), dtype=np.uint8)
    for k, v in extra.items():
        out["x_" + k] = np.asarray(v)
    np.savez_compressed(path, **out)


def load(path) -> tuple[R.FlatScene, R.CRenderDesc, dict]:
    z = np.load(path)
    kw = {}
    for k in _ARRAYS:
        kw[k] = np.ascontiguousarray(z["a_" + k]) if "a_" + k in z else None
    for k, ctype in _RECORDS.items():
        if "r_" + k in z:
            n = int(z["n_" + k])
            kw[k] = (ctype * n).from_buffer_copy(z["r_" + k].tobytes())
        else:
            kw[k] = None
    flat = R.FlatScene(scene_radius=float(z["scene_radius"]), **kw)
    desc = R.CRenderDesc.from_buffer_copy(z["desc"].tobytes())
    extra = {k[2:]: z[k] for k in z.files if k.startswith("x_")}
    return flat, desc, extra


def equal(a: R.FlatScene, b: R.FlatScene) -> bool:
    for k in _ARRAYS:
        x, y = getattr(a, k), getattr(b, k)
        if (x is None) != (y is None):
            return False
        if x is not None and not np.array_equal(np.asarray(x), np.asarray(y)):
            return False
    for k in _RECORDS:
        x, y = getattr(a, k), getattr(b, k)
        if bytes(x if x is not None else b"") != bytes(y if y is not None else b""):
            return False
    return np.float32(a.scene_radius) == np.float32(b.scene_radius)  # a float in the C ABI
