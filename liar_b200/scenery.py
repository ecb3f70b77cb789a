"""Scene objects of the scene API (``liar.scenery``, src/liar/scenery/). They record geometry and
shaders; RenderEngine flattens them into one triangle soup for the GPU."""
from __future__ import annotations

import numpy as np

from .textures import Constant


class SceneObject:
    def __init__(self):
        self.shader = None
        self.interior = None


class List(SceneObject):
    """Group of children (scenery/list.cpp); the tree variants only change how the reference
    finds the nearest child, which the GPU tree over the whole soup replaces."""

    def __init__(self, children=()):
        super().__init__()
        self.children = list(children)

    def add(self, child):
        self.children.append(child)


class QbvhTree(List):
    pass


class AabbTree(List):
    pass


class AabpTree(List):
    pass


class OctTree(List):
    pass


class Parallelogram(SceneObject):
    def __init__(self, support, sizeU, sizeV):
        super().__init__()
        self.support = tuple(float(x) for x in support)
        self.sizeU = tuple(float(x) for x in sizeU)
        self.sizeV = tuple(float(x) for x in sizeV)

    def triangles(self):
        s, u, v = (np.asarray(x, dtype=np.float64) for x in (self.support, self.sizeU, self.sizeV))
        verts = np.stack([s, s + u, s + u + v, s + v]).astype(np.float32)
        return verts, np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32), None, None

    def corner_uvs(self):
        """The parametric (u, v) of support + u sizeU + v sizeV at the corners (parallelogram.cpp:77-89)."""
        return np.array([[[0, 0], [1, 0], [1, 1]], [[0, 0], [1, 1], [0, 1]]], dtype=np.float32)

    @property
    def area(self) -> float:
        return float(np.linalg.norm(np.cross(self.sizeU, self.sizeV)))


class Triangle(SceneObject):
    def __init__(self, a, b, c):
        super().__init__()
        self.vertices = (tuple(a), tuple(b), tuple(c))

    def triangles(self):
        return np.asarray(self.vertices, dtype=np.float32), np.array([[0, 1, 2]], dtype=np.uint32), None, None


class TriangleMesh(SceneObject):
    """TriangleMesh(vertices, normals, uvs, triangles) (scenery/triangle_mesh.cpp). A triangle is
    three vertex indices, or three (vertex, normal[, uv]) index tuples."""

    def __init__(self, vertices, normals=(), uvs=(), triangles=()):
        super().__init__()
        self.vertices = np.asarray(vertices, dtype=np.float32).reshape(-1, 3)
        self.normals = np.asarray(normals, dtype=np.float32).reshape(-1, 3) if len(normals) else None
        self.uvs = uvs
        tri = list(triangles) if not isinstance(triangles, np.ndarray) else triangles
        if isinstance(tri, np.ndarray) and tri.ndim == 2:
            self._vi = tri.astype(np.uint32)
            self._ni = None
            self._ti = None
        else:
            vi, ni, ti = [], [], []
            has_n = has_t = False
            for t in tri:
                row_v, row_n, row_t = [], [], []
                for c in t:
                    if isinstance(c, (tuple, list)):
                        row_v.append(int(c[0]))
                        n = int(c[1]) if len(c) > 1 and c[1] is not None else -1
                        u = int(c[2]) if len(c) > 2 and c[2] is not None else -1
                        row_n.append(n)
                        row_t.append(u)
                        has_n |= n >= 0
                        has_t |= u >= 0
                    else:
                        row_v.append(int(c))
                        row_n.append(-1)
                        row_t.append(-1)
                vi.append(row_v)
                ni.append(row_n)
                ti.append(row_t)
            self._vi = np.asarray(vi, dtype=np.uint32).reshape(-1, 3)
            self._ni = np.asarray(ni, dtype=np.int32).reshape(-1, 3) if has_n else None
            self._ti = np.asarray(ti, dtype=np.int32).reshape(-1, 3) if has_t else None

    def triangles(self):
        return self.vertices, self._vi, self.normals, self._ni

    def corner_uvs(self):
        """The corners' uvs of triangles that index them; a triangle without has the barycentric
        coordinates of the hit as its uv (corners (0, 0), (1, 0), (0, 1))."""
        if self._ti is None or len(self.uvs) == 0:
            return None
        table = np.asarray(self.uvs, dtype=np.float32).reshape(-1, 2)
        if (self._ti >= len(table)).any():
            raise IndexError("TriangleMesh: uv index out of range")
        bary = np.array([[0, 0], [1, 0], [0, 1]], dtype=np.float32)
        full = (self._ti >= 0).all(axis=1, keepdims=True)[..., None]
        return np.where(full, table[np.maximum(self._ti, 0)], bary[None]).astype(np.float32)


class Sphere(SceneObject):
    """Sphere(center, radius) (scenery/sphere.cpp): an analytic sphere, intersected exactly on
    the GPU. With ``subdivisions`` it is flattened into a geodesic triangle mesh with exact normals
    instead; a sphere that is an area light's surface, or that sits under a transformation that is
    not a similarity, always is (with 5 subdivisions unless given)."""

    def __init__(self, center=(0, 0, 0), radius=1.0, subdivisions: int | None = None):
        super().__init__()
        self.center = tuple(float(x) for x in center)
        self.radius = float(radius)
        self.subdivisions = None if subdivisions is None else int(subdivisions)

    @property
    def analytic(self) -> bool:
        return self.subdivisions is None

    def triangles(self):
        from .scenes import icosahedron, subdivide
        v, f = icosahedron()
        for _ in range(self.subdivisions if self.subdivisions is not None else 5):
            v, f = subdivide(v, f)
        verts = (v * self.radius + np.asarray(self.center)).astype(np.float32)
        return verts, f.astype(np.uint32), v.astype(np.float32), f.astype(np.int32)

    def corner_uvs(self):
        """(phi / 2 pi, theta / pi) of the corners' normals (sphere.cpp:130-152), phi unwrapped per
        triangle across the seam and taken from the other corners at the poles."""
        from .scenes import icosahedron, subdivide
        v, f = icosahedron()
        for _ in range(self.subdivisions if self.subdivisions is not None else 5):
            v, f = subdivide(v, f)
        n = v / np.linalg.norm(v, axis=1, keepdims=True)
        u = np.arctan2(n[:, 1], n[:, 0]) / (2 * np.pi)
        w = np.arccos(np.clip(n[:, 2], -1.0, 1.0)) / np.pi
        cu, cw = u[f], w[f]                                   # n_tris x 3
        cu = np.where(cu < cu.max(axis=1, keepdims=True) - 0.5, cu + 1.0, cu)
        pole = np.hypot(n[:, 0], n[:, 1])[f] < 1e-6
        if pole.any():
            other = np.where(pole, np.nan, cu)
            fill = np.nanmean(other, axis=1, keepdims=True)
            cu = np.where(pole, fill, cu)
        return np.stack([cu, cw], axis=-1).astype(np.float32)


class Box(SceneObject):
    """Box(), Box((min, max)) or Box(min, max) (scenery/box.cpp; the default is [-1, 1]^3),
    flattened into 12 outward-wound triangles."""

    def __init__(self, *args):
        super().__init__()
        if not args:
            lo, hi = (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0)
        elif len(args) == 1:
            lo, hi = args[0]
        elif len(args) == 2:
            lo, hi = args
        else:
            raise TypeError("Box(), Box((min, max)) or Box(min, max)")
        self.min = tuple(float(x) for x in lo)
        self.max = tuple(float(x) for x in hi)

    @property
    def bounds(self):
        return (self.min, self.max)

    @bounds.setter
    def bounds(self, value):
        self.min, self.max = (tuple(float(x) for x in v) for v in value)

    def triangles(self):
        lo, hi = np.asarray(self.min, dtype=np.float64), np.asarray(self.max, dtype=np.float64)
        # corner k = (x bit 0, y bit 1, z bit 2)
        corners = np.array([[hi[0] if k & 1 else lo[0], hi[1] if k & 2 else lo[1], hi[2] if k & 4 else lo[2]]
                            for k in range(8)], dtype=np.float32)
        quads = [(0, 4, 6, 2), (1, 3, 7, 5),   # -x, +x
                 (0, 1, 5, 4), (2, 6, 7, 3),   # -y, +y
                 (0, 2, 3, 1), (4, 5, 7, 6)]   # -z, +z
        tris = []
        for a, b, c, d in quads:
            tris += [(a, b, c), (a, c, d)]
        return corners, np.asarray(tris, dtype=np.uint32), None, None

    def corner_uvs(self):
        """Box::doLocalContext (box.cpp:216-250): on the face of axis k, u and v run over the
        axes k + 1 and k + 2 from the minimum, v mirrored on the faces that look down the axis."""
        corners, tris, _, _ = self.triangles()
        lo, size = np.asarray(self.min, dtype=np.float64), np.asarray(self.max, dtype=np.float64) - np.asarray(self.min)
        out = np.zeros((len(tris), 3, 2), dtype=np.float32)
        for k, t in enumerate(tris):
            axis = k // 4
            positive = (k // 2) % 2 == 1
            i, j = (axis + 1) % 3, (axis + 2) % 3
            for c in range(3):
                p = corners[t[c]].astype(np.float64)
                uu = (p[i] - lo[i]) / size[i] if size[i] else 0.0
                vv = (p[j] - lo[j]) / size[j] if size[j] else 0.0
                out[k, c] = (uu, vv if positive else 1.0 - vv)
        return out


def as_matrix(m) -> np.ndarray:
    """A 4 x 4 float64 affine matrix from a 4 x 4 or 3 x 4 nested sequence (row-major, the last
    column the translation), 16 or 12 numbers, or an object with a `matrix` attribute."""
    if hasattr(m, "matrix"):
        m = m.matrix
    a = np.asarray(m, dtype=np.float64)
    if a.size == 16:
        a = a.reshape(4, 4)
    elif a.size == 12:
        a = np.vstack([a.reshape(3, 4), [0.0, 0.0, 0.0, 1.0]])
    else:
        raise ValueError("a transformation is a 4 x 4 or 3 x 4 matrix")
    if not np.allclose(a[3], [0.0, 0.0, 0.0, 1.0]):
        raise ValueError("only affine transformations are supported (last row 0, 0, 0, 1)")
    return a


class Transformation(SceneObject):
    """Transformation(child, localToWorld) (scenery/transformation.cpp): the child in a local frame.
    The flattening applies localToWorld to the child's vertices and light geometry and the inverse
    transpose to its normals."""

    def __init__(self, child, localToWorld):
        super().__init__()
        self.child = child
        self.localToWorld = localToWorld

    @property
    def localToWorld(self) -> np.ndarray:
        return self._m

    @localToWorld.setter
    def localToWorld(self, m):
        a = as_matrix(m)
        if abs(np.linalg.det(a[:3, :3])) < 1e-300:
            raise ValueError("singular transformation")
        self._m = a

    @property
    def worldToLocal(self) -> np.ndarray:
        return np.linalg.inv(self._m)

    def matrix(self) -> np.ndarray:
        return self._m


class Translation(SceneObject):
    """Translation(child, offset) (scenery/translation.cpp): localToWorld is the offset vector."""

    def __init__(self, child, localToWorld=(0.0, 0.0, 0.0)):
        super().__init__()
        self.child = child
        self.localToWorld = localToWorld

    @property
    def localToWorld(self):
        return self._t

    @localToWorld.setter
    def localToWorld(self, v):
        self._t = tuple(float(x) for x in v)

    @property
    def worldToLocal(self):
        return tuple(-x for x in self._t)

    def matrix(self) -> np.ndarray:
        a = np.eye(4)
        a[:3, 3] = self._t
        return a


class SceneLight(SceneObject):
    pass


class LightArea(SceneLight):
    """LightArea(surface) (scenery/light_area.cpp): a surface that emits radiance."""

    def __init__(self, surface, radiance=None):
        super().__init__()
        self.surface = surface
        self.radiance = radiance if radiance is not None else Constant(1.0).value
        self.numberOfEmissionSamples = 9
        self.isDoubleSided = False


class LightPoint(SceneLight):
    def __init__(self, position=(0, 0, 0), intensity=None):
        super().__init__()
        self.position = tuple(float(x) for x in position)
        self.intensity = intensity if intensity is not None else Constant(1.0).value
        self.numberOfEmissionSamples = 1


class LightSky(SceneLight):
    """Constant-radiance sky at a fixed distance of 1000 scene radii (scenery/light_sky.cpp)."""

    def __init__(self, radiance=None):
        super().__init__()
        self.radiance = radiance if radiance is not None else Constant(1.0)
        self.numberOfEmissionSamples = 1
