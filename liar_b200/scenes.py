"""Seeded synthetic scenes of the benchmark configurations (no dataset is involved).

* :func:`displaced_icosphere` -- the traversal workload: an icosahedron subdivided ``levels``
  times (8 -> 20 * 4**8 = 1,310,720 triangles, 655,362 vertices), vertices on the unit sphere
  displaced radially by ``r = 1 + amplitude * fbm(p)`` with 4 octaves of gradient noise
  (lacunarity 2, gain 0.5). The noise is improved Perlin noise (K. Perlin, "Improving noise",
  SIGGRAPH 2002: quintic fade, 12 edge gradients padded to 16) with a permutation drawn from
  numpy's PCG64 with the given seed -- the same family as the reference's Perlin/FBm textures
  (src/liar/textures/perlin.cpp, src/liar/textures/fbm.cpp), not the same table.
* :func:`random_rays` -- origins uniform in the mesh's bounding box scaled 1.5x about its centre,
  directions uniform on the sphere (z = 1 - 2u, phi = 2 pi v), PCG64 with the given seed.
"""
from __future__ import annotations

import numpy as np


def icosahedron() -> tuple[np.ndarray, np.ndarray]:
    p = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([[-1, p, 0], [1, p, 0], [-1, -p, 0], [1, -p, 0], [0, -1, p], [0, 1, p], [0, -1, -p], [0, 1, -p],
                  [p, 0, -1], [p, 0, 1], [-p, 0, -1], [-p, 0, 1]], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    return v, f


def subdivide(v: np.ndarray, f: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """One midpoint subdivision, new vertices projected to the unit sphere."""
    e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]], axis=0)
    e.sort(axis=1)
    key = e[:, 0] * (v.shape[0] + 1) + e[:, 1]
    uniq, inv = np.unique(key, return_inverse=True)
    a = uniq // (v.shape[0] + 1)
    b = uniq % (v.shape[0] + 1)
    mid = v[a] + v[b]
    mid /= np.linalg.norm(mid, axis=1, keepdims=True)
    base = v.shape[0]
    m = inv.reshape(3, -1) + base  # midpoints of edges (0,1), (1,2), (2,0) per face
    m01, m12, m20 = m[0], m[1], m[2]
    nf = np.concatenate([
        np.stack([f[:, 0], m01, m20], axis=1),
        np.stack([f[:, 1], m12, m01], axis=1),
        np.stack([f[:, 2], m20, m12], axis=1),
        np.stack([m01, m12, m20], axis=1),
    ], axis=0)
    return np.concatenate([v, mid], axis=0), nf


_GRAD = np.array([[1, 1, 0], [-1, 1, 0], [1, -1, 0], [-1, -1, 0], [1, 0, 1], [-1, 0, 1], [1, 0, -1], [-1, 0, -1],
                  [0, 1, 1], [0, -1, 1], [0, 1, -1], [0, -1, -1], [1, 1, 0], [-1, 1, 0], [0, -1, 1], [0, -1, -1]],
                 dtype=np.float64)


def perlin_noise(p: np.ndarray, perm: np.ndarray) -> np.ndarray:
    """Improved gradient noise at points p (n, 3); perm is a 512-entry doubled permutation."""
    fl = np.floor(p)
    i = fl.astype(np.int64) & 255
    x = p - fl

    def fade(t):
        return t * t * t * (t * (t * 6.0 - 15.0) + 10.0)

    u = fade(x)
    out = np.zeros(p.shape[0])
    acc = {}
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                h = perm[perm[perm[i[:, 0] + dx] + i[:, 1] + dy] + i[:, 2] + dz] & 15
                g = _GRAD[h]
                d = x - np.array([dx, dy, dz], dtype=np.float64)
                acc[(dx, dy, dz)] = np.einsum("ij,ij->i", g, d)
    lerp = lambda a, b, t: a + t * (b - a)  # noqa: E731
    x00 = lerp(acc[(0, 0, 0)], acc[(1, 0, 0)], u[:, 0])
    x10 = lerp(acc[(0, 1, 0)], acc[(1, 1, 0)], u[:, 0])
    x01 = lerp(acc[(0, 0, 1)], acc[(1, 0, 1)], u[:, 0])
    x11 = lerp(acc[(0, 1, 1)], acc[(1, 1, 1)], u[:, 0])
    out = lerp(lerp(x00, x10, u[:, 1]), lerp(x01, x11, u[:, 1]), u[:, 2])
    return out


def fbm(p: np.ndarray, seed: int = 0, octaves: int = 4, lacunarity: float = 2.0, gain: float = 0.5) -> np.ndarray:
    rng = np.random.default_rng(seed)
    perm = rng.permutation(256)
    perm = np.concatenate([perm, perm]).astype(np.int64)
    out = np.zeros(p.shape[0])
    freq, amp = 1.0, 1.0
    for _ in range(octaves):
        out += amp * perlin_noise(p * freq, perm)
        freq *= lacunarity
        amp *= gain
    return out


def displaced_icosphere(levels: int = 8, amplitude: float = 0.05, seed: int = 0, octaves: int = 4,
                        center=(0.0, 0.0, 0.0), radius: float = 1.0) -> tuple[np.ndarray, np.ndarray]:
    """Returns float32 vertices (n, 3) and uint32 triangles (m, 3)."""
    v, f = icosahedron()
    for _ in range(levels):
        v, f = subdivide(v, f)
    r = 1.0 + amplitude * fbm(v, seed=seed, octaves=octaves)
    v = v * (radius * r)[:, None] + np.asarray(center, dtype=np.float64)
    return v.astype(np.float32), f.astype(np.uint32)


def random_rays(vertices: np.ndarray, n: int, seed: int = 0, tmin: float = 0.0, tmax: float = np.inf,
                scale: float = 1.5) -> np.ndarray:
    """(n, 8) float32 rays: origins uniform in the bbox scaled ``scale`` about its centre,
    unit directions uniform on the sphere."""
    lo = vertices.min(axis=0).astype(np.float64)
    hi = vertices.max(axis=0).astype(np.float64)
    c = 0.5 * (lo + hi)
    h = 0.5 * scale * (hi - lo)
    rng = np.random.default_rng(seed)
    out = np.empty((n, 8), dtype=np.float32)
    chunk = 1 << 22
    for s in range(0, n, chunk):
        m = min(chunk, n - s)
        o = c + (rng.random((m, 3)) * 2.0 - 1.0) * h
        u = rng.random(m)
        w = rng.random(m)
        z = 1.0 - 2.0 * u
        rr = np.sqrt(np.maximum(0.0, 1.0 - z * z))
        phi = 2.0 * np.pi * w
        out[s:s + m, 0:3] = o
        out[s:s + m, 3] = tmin
        out[s:s + m, 4] = rr * np.cos(phi)
        out[s:s + m, 5] = rr * np.sin(phi)
        out[s:s + m, 6] = z
        out[s:s + m, 7] = tmax
    return out
