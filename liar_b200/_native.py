"""ctypes binding of the sm_100a library ``libliar_gpu.so`` (C ABI in include/liar_gpu.h).

There is no CPU fallback: importing this module raises if the library has not been built, and
every entry point raises :class:`LiarGpuError` with the library's message when it fails.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("LIAR_GPU_LIB", _HERE / "libliar_gpu.so"))

LIAR_OK = 0
STATUS_NAMES = {
    -1: "LIAR_ERR_INVALID",
    -2: "LIAR_ERR_CUDA",
    -3: "LIAR_ERR_NO_DEVICE",
    -4: "LIAR_ERR_OOM",
    -5: "LIAR_ERR_STACK",
    -6: "LIAR_ERR_TIMEOUT",
    -7: "LIAR_ERR_CANCELLED",
    -8: "LIAR_ERR_UNSUPPORTED",
}


class LiarGpuError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {message}")
        self.code = code


class Ray(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("ox", "oy", "oz", "tmin", "dx", "dy", "dz", "tmax")]


class Hit(C.Structure):
    _fields_ = [("prim", C.c_int32), ("t", C.c_float)]


class BuildOpts(C.Structure):
    _fields_ = [("max_leaf_size", C.c_int), ("sah_bins", C.c_int), ("traversal_cost", C.c_float), ("threads", C.c_int)]


class TraceConfig(C.Structure):
    _fields_ = [("block_size", C.c_int), ("smem_stack", C.c_int)]


class MeshStats(C.Structure):
    _fields_ = [
        ("n_triangles", C.c_uint64),
        ("n_nodes", C.c_uint64),
        ("n_leaves", C.c_uint64),
        ("max_depth", C.c_uint32),
        ("stack_needed", C.c_uint32),
        ("sah_cost", C.c_double),
        ("device_bytes", C.c_uint64),
        ("build_seconds", C.c_double),
    ]


_vp = C.c_void_p
_sz = C.c_size_t

# name -> (restype, argtypes); every symbol declared in include/liar_gpu.h is listed here
SIGNATURES: dict[str, tuple] = {
    "liar_gpu_abi_version": (C.c_int, []),
    "liar_gpu_create": (C.c_int, [C.POINTER(_vp), C.c_int]),
    "liar_gpu_destroy": (None, [_vp]),
    "liar_gpu_last_error": (C.c_char_p, [_vp]),
    "liar_gpu_set_stream": (C.c_int, [_vp, _vp]),
    "liar_gpu_synchronize": (C.c_int, [_vp]),
    "liar_gpu_set_cancel_flag": (C.c_int, [_vp, _vp]),
    "liar_gpu_set_fault_test": (C.c_int, [_vp, C.c_int]),
    "liar_gpu_set_trace_config": (C.c_int, [_vp, C.POINTER(TraceConfig)]),
    "liar_gpu_get_trace_config": (C.c_int, [_vp, C.POINTER(TraceConfig)]),
    "liar_gpu_mesh_build": (C.c_int, [_vp, _vp, _sz, _vp, _sz, _vp, C.POINTER(_vp)]),
    "liar_gpu_mesh_destroy": (None, [_vp]),
    "liar_gpu_mesh_stats": (C.c_int, [_vp, C.POINTER(MeshStats)]),
    "liar_gpu_trace": (C.c_int, [_vp, _vp, _vp, _sz, _vp, C.c_int]),
    "liar_gpu_trace_device": (C.c_int, [_vp, _vp, _vp, _sz, _vp, C.c_int, _vp]),
    "liar_gpu_trace_counted_device": (C.c_int, [_vp, _vp, _vp, _sz, _vp, C.c_int, _vp, _vp]),
    "liar_gpu_trace_device_noalloc": (C.c_int, [_vp, _vp, _sz, _vp, C.c_int, _vp]),
    # renderer (liar_b200/render.py rebinds these with its struct types)
    "liar_gpu_scene_upload": (C.c_int, [_vp, _vp, C.POINTER(_vp)]),
    "liar_gpu_scene_destroy": (None, [_vp]),
    "liar_gpu_render": (C.c_int, [_vp, _vp, _vp, _vp]),
    "liar_gpu_render_device": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "liar_gpu_render_stats": (C.c_int, [_vp, _vp]),
    # photon maps (liar_b200/photons.py)
    "liar_gpu_photon_map_build": (C.c_int, [_vp, _vp, _sz, C.c_float, C.POINTER(_vp)]),
    "liar_gpu_photon_map_build_device": (C.c_int, [_vp, _vp, _sz, C.c_float, C.POINTER(_vp), _vp]),
    "liar_gpu_photon_map_rebuild_device": (C.c_int, [_vp, _vp, _vp, _sz, C.c_float, _vp]),
    "liar_gpu_photon_map_destroy": (None, [_vp]),
    "liar_gpu_photon_gather": (C.c_int, [_vp, _vp, _vp, _sz, C.c_int, _vp, _vp, _vp]),
    "liar_gpu_photon_gather_device": (C.c_int, [_vp, _vp, _vp, _sz, C.c_int, _vp, _vp, _vp, _vp]),
    "liar_gpu_photon_trace": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "liar_gpu_photon_mapper_stats": (C.c_int, [_vp, _vp, _vp]),
    "liar_gpu_photon_mapper_get_map": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, _vp, _vp, C.c_size_t, _vp]),
    "liar_gpu_photon_mapper_get_irradiance": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_size_t, _vp]),
    "liar_gpu_set_recovery": (C.c_int, [_vp, _vp, C.c_int, _vp, _vp, C.c_int, _vp, C.c_int]),
    "liar_gpu_recovery_locate_device": (C.c_int, [_vp, _vp, C.c_size_t, _vp, _vp, _vp]),
    "liar_gpu_photon_estimate_device": (C.c_int, [_vp, _vp, _vp, _sz, _vp, _sz, C.c_int, _vp, _vp, _vp, C.c_float,
                                                  _vp, _vp]),
    # batched rendering (liar_b200/batch.py)
    "liar_gpu_batch_create": (C.c_int, [_vp, _vp, _sz, _vp, C.POINTER(_vp)]),
    "liar_gpu_batch_launch": (C.c_int, [_vp, _vp, _vp]),
    "liar_gpu_batch_stats": (C.c_int, [_vp, _vp]),
    "liar_gpu_batch_destroy": (None, [_vp]),
    # learned path guiding (liar_b200/guiding.py)
    "liar_gpu_guide_create": (C.c_int, [_vp, _vp, C.POINTER(_vp)]),
    "liar_gpu_guide_destroy": (None, [_vp]),
    "liar_gpu_guide_param_count": (_sz, []),
    "liar_gpu_guide_get_params": (C.c_int, [_vp, _vp, _vp, _sz]),
    "liar_gpu_guide_set_params": (C.c_int, [_vp, _vp, _vp, _sz]),
    "liar_gpu_guide_eval_device": (C.c_int, [_vp, _vp, _vp, _sz, _vp, _vp]),
    "liar_gpu_guide_train_device": (C.c_int, [_vp, _vp, _vp, _sz, C.c_int, _vp, _vp, _vp]),
    "liar_gpu_guide_sample_device": (C.c_int, [_vp, _vp, _vp, _sz, _vp, _vp, _vp]),
    "liar_gpu_guide_stats": (C.c_int, [_vp, _vp]),
    "liar_gpu_render_guided_device": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, _vp, _vp]),
    "liar_gpu_render_guided_stats": (C.c_int, [_vp, _vp]),
}


def load(path: Path | str | None = None) -> C.CDLL:
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(
            f"{p} is missing: build it with `python -m liar_b200.build` (there is no CPU fallback)"
        )
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_LIB: C.CDLL | None = None


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = load()
    return _LIB


def check(code: int, ctx=None) -> None:
    if code != LIAR_OK:
        msg = lib().liar_gpu_last_error(ctx).decode(errors="replace") if ctx else ""
        raise LiarGpuError(code, msg)
