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
    "liar_gpu_photon_map_rebuild_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_float,
                                                     C.c_void_p]),
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

    def rebuild(self, device_ptr: int, n: int, r_max: float | None = None, stream: int | None = None):
        """Builds the map again over n device positions, in its existing buffers (grown when needed)."""
        r = self.r_max if r_max is None else float(r_max)
        self.ctx.check(self.ctx._lib.liar_gpu_photon_map_rebuild_device(self.ctx.handle, self.handle,
                                                                        C.c_void_p(device_ptr), int(n), r,
                                                                        C.c_void_p(stream or 0)))
        self.n, self.r_max = int(n), r

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


# ---- photon tracing (liar_gpu_photon_trace)

class PhotonDesc(C.Structure):
    _fields_ = [("max_ray_generation", C.c_int32), ("ray_traced_direct", C.c_int32), ("seed", C.c_uint64),
                ("global_target", C.c_uint64), ("max_emitted", C.c_uint64), ("wave", C.c_uint64),
                ("final_gather", C.c_int32), ("caustics_quality", C.c_float)]


class PhotonBuffers(C.Structure):
    _fields_ = [("position", C.c_void_p), ("omega_in", C.c_void_p), ("power", C.c_void_p), ("path", C.c_void_p),
                ("tag", C.c_void_p), ("capacity", C.c_uint64), ("normal", C.c_void_p)]


class PhotonCounts(C.Structure):
    _fields_ = [("stored", C.c_uint64), ("global_", C.c_uint64), ("caustic", C.c_uint64), ("emitted", C.c_uint64)]


GLOBAL, CAUSTIC = 1, 2


def photon_desc(global_target: int, max_emitted: int = 100_000_000, max_ray_generation: int = 8, seed: int = 0,
                wave: int = 0, ray_traced_direct: bool = True, final_gather: bool = False,
                caustics_quality: float = 1.0) -> PhotonDesc:
    """liar_photon_desc; caustics_quality is PhotonMapper.causticsQuality (storage probabilities
    1 / max(q, 1) for the global map and q / max(q, 1) for the caustic map; stored powers are not
    divided by them)."""
    d = PhotonDesc()
    q = max(float(caustics_quality), 0.0)
    d.caustics_quality = q if q > 0.0 else -1.0
    d.max_ray_generation = int(max_ray_generation)
    d.ray_traced_direct = int(bool(ray_traced_direct))
    d.seed = int(seed)
    d.global_target = int(global_target)
    d.max_emitted = int(max_emitted)
    d.wave = int(wave)
    d.final_gather = int(bool(final_gather))
    return d


def trace_photons(gpu_scene, desc: PhotonDesc, capacity: int, stream: int | None = None):
    """Runs PhotonMapper::fillPhotonMaps on the GPU. Returns (dict of torch device tensors, counts)."""
    import torch
    ctx = gpu_scene.ctx
    lib = ctx._lib
    fn = lib.liar_gpu_photon_trace
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(PhotonDesc), C.POINTER(PhotonBuffers), C.POINTER(PhotonCounts),
                   C.c_void_p]
    dev = f"cuda:{ctx.device}"
    buf = {
        "position": torch.empty((capacity, 3), dtype=torch.float32, device=dev),
        "omega_in": torch.empty((capacity, 3), dtype=torch.float32, device=dev),
        "power": torch.empty((capacity, 3), dtype=torch.float32, device=dev),
        "path": torch.empty(capacity, dtype=torch.int32, device=dev),
        "tag": torch.empty(capacity, dtype=torch.int32, device=dev),
    }
    b = PhotonBuffers(*(buf[k].data_ptr() for k in ("position", "omega_in", "power", "path", "tag")), int(capacity))
    counts = PhotonCounts()
    torch.cuda.synchronize()
    ctx.check(fn(ctx.handle, gpu_scene.handle, C.byref(desc), C.byref(b), C.byref(counts), C.c_void_p(stream or 0)))
    n = int(counts.stored)
    out = {k: v[:n] for k, v in buf.items()}
    return out, {"stored": n, "global": int(counts.global_), "caustic": int(counts.caustic),
                 "emitted": int(counts.emitted)}


def automatic_radius(power_xyz: np.ndarray, emitted: int, estimation_size: int = 50, tolerance: float = 0.05) -> float:
    """PhotonMapper::buildPhotonMap's automatic estimation radius (photon_mapper.cpp:815-833): the
    median photon power (|X|+|Y|+|Z| after scaling by 1 / photons emitted) sets the area."""
    p = np.abs(np.asarray(power_xyz, dtype=np.float64)).sum(axis=1) / max(emitted, 1)
    median = float(p[len(p) // 2]) if len(p) else 0.0
    area = estimation_size * median / tolerance
    return float(np.sqrt(area) / np.pi)
