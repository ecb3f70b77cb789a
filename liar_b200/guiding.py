"""Learned path guiding: the guide network (liar_gpu_guide_*) and the guided renderer
(liar_gpu_render_guided_device), include/liar_gpu.h.

No reference counterpart: the reference's AdjointPhotonTracer samples BSDF and lights only
(src/liar/tracers/adjoint_photon_tracer.cpp:212-292). Device buffers are torch tensors.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

INPUTS, MIXTURE, RECORD = 9, 40, 13


class GuideConfig(C.Structure):
    _fields_ = [("bounds_lo", C.c_float * 3), ("bounds_hi", C.c_float * 3), ("learning_rate", C.c_float),
                ("guide_probability", C.c_float), ("light_probability", C.c_float), ("batch_records", C.c_int32),
                ("steps_per_pass", C.c_int32),
                ("seed", C.c_uint64)]


def scene_bounds(flat, margin: float = 1e-3) -> tuple[np.ndarray, np.ndarray]:
    """The box of a flattened scene's vertices, grown by margin x its diagonal."""
    lo = flat.vertices.min(axis=0).astype(np.float64)
    hi = flat.vertices.max(axis=0).astype(np.float64)
    pad = margin * float(np.linalg.norm(hi - lo)) + 1e-6
    return (lo - pad).astype(np.float32), (hi + pad).astype(np.float32)


def _ptr(t) -> int:
    return t.data_ptr() if hasattr(t, "data_ptr") else int(t)


CUDA_STREAM_LEGACY = 1  # the handle value of cudaStreamLegacy


def _stream(stream) -> C.c_void_p:
    """The given stream, else torch's current stream (device tensors are produced and consumed
    there; torch's default stream is the legacy default stream, which NULL would not select)."""
    if stream is None:
        import torch
        stream = torch.cuda.current_stream().cuda_stream or CUDA_STREAM_LEGACY
    return C.c_void_p(stream)


class Guide:
    def __init__(self, ctx, bounds, learning_rate: float = 0.0, guide_probability: float = 0.5,
                 batch_records: int = 0, steps_per_pass: int = 0, seed: int = 0, light_probability: float = 0.0):
        self.ctx = ctx
        c = GuideConfig()
        c.bounds_lo[:] = [float(x) for x in bounds[0]]
        c.bounds_hi[:] = [float(x) for x in bounds[1]]
        c.learning_rate = float(learning_rate)
        c.guide_probability = float(guide_probability)
        c.light_probability = float(light_probability)
        c.batch_records = int(batch_records)
        c.steps_per_pass = int(steps_per_pass)
        c.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        self.config = c
        h = C.c_void_p()
        ctx.check(ctx._lib.liar_gpu_guide_create(ctx.handle, C.byref(c), C.byref(h)))
        self.handle = h
        self.n_params = int(ctx._lib.liar_gpu_guide_param_count())

    def close(self):
        if getattr(self, "handle", None):
            self.ctx._lib.liar_gpu_guide_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> np.ndarray:
        out = np.zeros(self.n_params, np.float32)
        self.ctx.check(self.ctx._lib.liar_gpu_guide_get_params(self.ctx.handle, self.handle, out.ctypes.data, out.size))
        return out

    @params.setter
    def params(self, value) -> None:
        v = np.ascontiguousarray(value, dtype=np.float32)
        self.ctx.check(self.ctx._lib.liar_gpu_guide_set_params(self.ctx.handle, self.handle, v.ctypes.data, v.size))

    def eval(self, inputs, out=None, stream=None):
        """inputs: (n, 9) float32 cuda tensor -> (n, 40) mixtures."""
        import torch
        n = inputs.shape[0]
        if out is None:
            out = torch.empty((n, MIXTURE), dtype=torch.float32, device=inputs.device)
        self.ctx.check(self.ctx._lib.liar_gpu_guide_eval_device(self.ctx.handle, self.handle, _ptr(inputs), n,
                                                                _ptr(out), _stream(stream)))
        return out

    def train_device(self, records, apply: bool = True, loss=None, stream=None) -> None:
        """One training step over records ((n, 13) float32 cuda tensor) queued on `stream`, without a
        synchronize; the batch's loss is written to `loss` (a one-element cuda tensor) when given."""
        self.ctx.check(self.ctx._lib.liar_gpu_guide_train_device(
            self.ctx.handle, self.handle, _ptr(records), records.shape[0], int(apply), C.c_void_p(0),
            C.c_void_p(_ptr(loss) if loss is not None else 0), _stream(stream)))

    def train_step(self, records, apply: bool = True, want_grad: bool = False, stream=None):
        """records: (n, 13) float32 cuda tensor. Returns (loss, gradient or None) after a synchronize."""
        import torch
        dev = records.device
        loss = torch.zeros(1, dtype=torch.float32, device=dev)
        grad = torch.zeros(self.n_params, dtype=torch.float32, device=dev) if want_grad else None
        self.ctx.check(self.ctx._lib.liar_gpu_guide_train_device(
            self.ctx.handle, self.handle, _ptr(records), records.shape[0], int(apply),
            C.c_void_p(_ptr(grad) if grad is not None else 0), _ptr(loss), _stream(stream)))
        torch.cuda.synchronize(dev)
        return float(loss.item()), (grad.cpu().numpy() if grad is not None else None)

    def sample(self, mixtures, u, stream=None):
        import torch
        n = mixtures.shape[0]
        dirs = torch.empty((n, 3), dtype=torch.float32, device=mixtures.device)
        pdf = torch.empty(n, dtype=torch.float32, device=mixtures.device)
        self.ctx.check(self.ctx._lib.liar_gpu_guide_sample_device(self.ctx.handle, _ptr(mixtures), _ptr(u), n,
                                                                  _ptr(dirs), _ptr(pdf), _stream(stream)))
        return dirs, pdf

    def stats(self) -> dict:
        out = (C.c_ulonglong * 4)()
        self.ctx.check(self.ctx._lib.liar_gpu_guide_stats(self.handle, out))
        return {"steps": out[0], "records": out[1], "guided": out[2], "passes": out[3]}

    def render(self, scene, desc, film_ptr: int, train: bool = True, stream=None) -> None:
        """Adds desc.spp guided samples per pixel to the device film (H x W x 8 sums)."""
        self.ctx.check(self.ctx._lib.liar_gpu_render_guided_device(self.ctx.handle, scene.handle, self.handle,
                                                                   C.byref(desc), int(train), C.c_void_p(film_ptr),
                                                                   _stream(stream)))


def render_stats(ctx) -> dict:
    out = (C.c_ulonglong * 4)()
    ctx.check(ctx._lib.liar_gpu_render_guided_stats(ctx.handle, out))
    return {"paths": out[0], "segments": out[1], "hits": out[2], "guided": out[3]}
