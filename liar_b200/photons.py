"""Photon maps on the GPU: build a hash grid over photon positions and gather the k nearest
photons within r_max for query points (the reference's KdTree<Photon>::rangeSearch, used by
PhotonMapper, src/liar/tracers/photon_mapper.cpp:798-835, 1254-1381)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N

_SIGS = {
    "liar_gpu_photon_map_build": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_float, C.POINTER(C.c_void_p)]),
    "liar_gpu_photon_map_build_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_float,
                                                   C.POINTER(C.c_void_p), C.c_void_p]),
    "liar_gpu_photon_map_destroy": (None, [C.c_void_p]),
    "liar_gpu_photon_gather": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_int, C.c_void_p,
                                         C.c_void_p, C.c_void_p]),
    "liar_gpu_photon_gather_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_int, C.c_void_p,
                                                C.c_void_p, C.c_void_p, C.c_void_p]),
}


class PhotonMap:
    def __init__(self, ctx, positions=None, r_max: float = 0.1, device_ptr: int | None = None, n: int | None = None,
                 stream: int | None = None):
        self.ctx = ctx
        lib = ctx._lib
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
        h = C.c_void_p()
        if device_ptr is not None:
            ctx.check(lib.liar_gpu_photon_map_build_device(ctx.handle, C.c_void_p(device_ptr), int(n), float(r_max),
                                                           C.byref(h), C.c_void_p(stream or 0)))
            self.n = int(n)
        else:
            P = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
            ctx.check(lib.liar_gpu_photon_map_build(ctx.handle, P.ctypes.data, P.shape[0], float(r_max), C.byref(h)))
            self.n = P.shape[0]
        self.handle = h
        self.r_max = float(r_max)

    def gather(self, queries, k: int = 64):
        Q = np.ascontiguousarray(queries, dtype=np.float32).reshape(-1, 3)
        idx = np.empty((Q.shape[0], k), np.int32)
        d2 = np.empty((Q.shape[0], k), np.float32)
        cnt = np.empty(Q.shape[0], np.int32)
        self.ctx.check(self.ctx._lib.liar_gpu_photon_gather(self.ctx.handle, self.handle, Q.ctypes.data, Q.shape[0],
                                                            int(k), idx.ctypes.data, d2.ctypes.data, cnt.ctypes.data))
        return idx, d2, cnt

    def gather_device(self, q_ptr: int, nq: int, k: int, idx_ptr: int, d2_ptr: int, cnt_ptr: int | None,
                      stream: int | None = None) -> None:
        self.ctx.check(self.ctx._lib.liar_gpu_photon_gather_device(
            self.ctx.handle, self.handle, C.c_void_p(q_ptr), int(nq), int(k), C.c_void_p(idx_ptr),
            C.c_void_p(d2_ptr), C.c_void_p(cnt_ptr or 0), C.c_void_p(stream or 0)))

    def close(self):
        if getattr(self, "handle", None):
            self.ctx._lib.liar_gpu_photon_map_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
