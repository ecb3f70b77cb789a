"""Host-side wrapper of the triangle-mesh entry points (closest hit / any hit).

Mirrors the reference's TriangleMesh as a scene object that answers intersect / isIntersecting
queries (src/liar/scenery/triangle_mesh.cpp:291-330), but batched: one call traces a whole
array of rays on the GPU through the C ABI of include/liar_gpu.h.

Ray arrays are float32 ``(n, 8)``: origin xyz, tmin, direction xyz, tmax (the BoundedRay of
src/liar/kernel/bounded_ray.h). Hits come back as ``prim`` (int32, -1 on a miss) and ``t``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N


class Context:
    """One CUDA device and stream; not re-entrant (one per host thread)."""

    def __init__(self, device: int = 0):
        self._lib = N.lib()
        h = C.c_void_p()
        N.check(self._lib.liar_gpu_create(C.byref(h), int(device)))
        self.handle = h
        self.device = int(device)

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.liar_gpu_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_stream(self, stream_ptr: int | None) -> None:
        N.check(self._lib.liar_gpu_set_stream(self.handle, C.c_void_p(stream_ptr or 0)), self.handle)

    def set_cancel_flag(self, flag: C.c_int32 | None) -> None:
        """Renders on this context stop between waves and bounces once flag.value != 0 and raise
        LiarGpuError(LIAR_ERR_CANCELLED) (liar_gpu_set_cancel_flag). The caller keeps flag alive;
        None removes it."""
        self._cancel = flag
        N.check(self._lib.liar_gpu_set_cancel_flag(self.handle, C.byref(flag) if flag is not None else None),
                self.handle)

    @property
    def trace_config(self) -> tuple[int, int]:
        """(threads per block, shared-memory stack entries per lane) of the trace kernels."""
        c = N.TraceConfig()
        N.check(self._lib.liar_gpu_get_trace_config(self.handle, C.byref(c)), self.handle)
        return c.block_size, c.smem_stack

    @trace_config.setter
    def trace_config(self, value: tuple[int, int]) -> None:
        c = N.TraceConfig(int(value[0]), int(value[1]))
        N.check(self._lib.liar_gpu_set_trace_config(self.handle, C.byref(c)), self.handle)

    def synchronize(self) -> None:
        N.check(self._lib.liar_gpu_synchronize(self.handle), self.handle)

    def check(self, code: int) -> None:
        N.check(code, self.handle)


def _as_rays(rays: np.ndarray) -> np.ndarray:
    rays = np.ascontiguousarray(rays, dtype=np.float32)
    if rays.ndim != 2 or rays.shape[1] != 8:
        raise ValueError("rays must be an (n, 8) float32 array: ox, oy, oz, tmin, dx, dy, dz, tmax")
    return rays


class Mesh:
    """A triangle mesh with its 4-wide SAH tree resident on the device."""

    def __init__(self, ctx: Context, vertices: np.ndarray, triangles: np.ndarray, max_leaf_size: int = 4,
                 sah_bins: int = 32, traversal_cost: float = 1.0, threads: int = 0):
        self.ctx = ctx
        v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(triangles, dtype=np.uint32).reshape(-1, 3)
        opts = N.BuildOpts(int(max_leaf_size), int(sah_bins), float(traversal_cost), int(threads))
        h = C.c_void_p()
        ctx.check(ctx._lib.liar_gpu_mesh_build(ctx.handle, v.ctypes.data, v.shape[0], t.ctypes.data, t.shape[0],
                                               C.byref(opts), C.byref(h)))
        self.handle = h
        self.n_triangles = t.shape[0]

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.ctx._lib.liar_gpu_mesh_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stats(self) -> dict:
        s = N.MeshStats()
        self.ctx.check(self.ctx._lib.liar_gpu_mesh_stats(self.handle, C.byref(s)))
        return {name: getattr(s, name) for name, _ in N.MeshStats._fields_}

    def intersect(self, rays: np.ndarray, any_hit: bool = False) -> tuple[np.ndarray, np.ndarray]:
        """Traces host rays; returns (prim, t) host arrays."""
        rays = _as_rays(rays)
        hits = np.empty((rays.shape[0], 2), dtype=np.int32)
        self.ctx.check(self.ctx._lib.liar_gpu_trace(self.ctx.handle, self.handle, rays.ctypes.data, rays.shape[0],
                                                    hits.ctypes.data, int(bool(any_hit))))
        return hits[:, 0].copy(), hits[:, 1].view(np.float32).copy()

    def trace_into(self, rays_ptr: int, n: int, hits_ptr: int, any_hit: bool = False, stream: int | None = None,
                   counters_ptr: int | None = None) -> None:
        """Asynchronous device call on raw device pointers (e.g. torch ``data_ptr()``)."""
        lib = self.ctx._lib
        if counters_ptr:
            code = lib.liar_gpu_trace_counted_device(self.ctx.handle, self.handle, C.c_void_p(rays_ptr), int(n),
                                                     C.c_void_p(hits_ptr), int(bool(any_hit)),
                                                     C.c_void_p(counters_ptr), C.c_void_p(stream or 0))
        else:
            code = lib.liar_gpu_trace_device(self.ctx.handle, self.handle, C.c_void_p(rays_ptr), int(n),
                                             C.c_void_p(hits_ptr), int(bool(any_hit)), C.c_void_p(stream or 0))
        self.ctx.check(code)
