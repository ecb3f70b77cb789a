"""RenderEngine of the scene API (src/liar/kernel/render_engine.cpp:170-358).

``engine.render()`` flattens ``engine.scene`` (cached until the scene object changes), renders
``sampler.samplesPerPixel`` samples of every pixel of ``sampler.resolution`` on the GPU with
``engine.tracer`` and hands the resolved XYZ + alpha film to ``engine.target``.

Cancellation follows RenderEngine::isCanceling (render_engine.cpp:239-242, 294-297): while a
render runs, a watcher thread polls ``target.isCanceling()`` and raises the context's cancel flag
(liar_gpu_set_cancel_flag); the GPU work then stops between waves and bounces and ``render()``
returns without writing the target, as the reference's engine returns from a cancelled render.
"""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np

from . import render as R
from ._native import LiarGpuError
from .trace import Context

_CTX: Context | None = None
LIAR_ERR_CANCELLED = -7

# the reference's geometric tolerance (kernel/kernel_common.cpp:32); the GPU path is built for it
_TOLERANCE = 1e-6
_tolerance = _TOLERANCE


def tolerance() -> float:
    """liar.tolerance() (kernel/kernel_common.cpp:32-45)."""
    return _tolerance


def setTolerance(value: float) -> None:
    """liar.setTolerance(): recorded; RenderEngine.render refuses a value other than the default,
    because the GPU kernels' inRange test is compiled for tolerance 1e-6."""
    global _tolerance
    _tolerance = float(value)


def default_context() -> Context:
    global _CTX
    if _CTX is None:
        _CTX = Context(0)
    return _CTX


def _canceling(target) -> bool:
    fn = getattr(target, "isCanceling", None)
    return bool(fn()) if callable(fn) else False


class RenderEngine:
    def __init__(self):
        self.tracer = None
        self.sampler = None
        self.camera = None
        self.scene = None
        self.target = None
        self.numberOfThreads = 0  # accepted for script compatibility; the GPU decides parallelism
        self.seed = 0
        self._gpu_scene = None
        self._scene_key = None

    def _scene(self):
        key = id(self.scene)
        if self._gpu_scene is None or self._scene_key != key:
            self._gpu_scene = R.GpuScene(default_context(), R.flatten(self.scene))
            self._scene_key = key
        return self._gpu_scene

    def render(self, time: float = 0.0, bucket=None):
        if self.camera is None or self.tracer is None or self.scene is None or self.sampler is None:
            # the reference throws here (render_engine.cpp:172-193)
            raise RuntimeError("RenderEngine needs a camera, a tracer, a sampler and a scene before render()")
        if getattr(self.sampler, "progressive", False):
            raise NotImplementedError(f"{type(self.sampler).__name__} is a progressive sampler; the GPU path renders "
                                      "with Stratifier or LatinHypercube")
        if _tolerance != _TOLERANCE:
            raise NotImplementedError(f"setTolerance({_tolerance!r}): the GPU path is built for the default "
                                      f"tolerance {_TOLERANCE!r}")
        w, h = self.sampler.resolution
        from .output import film_settings
        desc = R.render_desc(self.camera, w, h, self.sampler.samplesPerPixel, self.tracer,
                             seed=self.seed or getattr(self.sampler, "seed_", 0), sampler=self.sampler.mode,
                             **film_settings(self.target))
        scene = self._scene()
        ctx = scene.ctx
        flag = C.c_int32(0)
        done = threading.Event()

        def watch():
            while not done.wait(0.02):
                if _canceling(self.target):
                    flag.value = 1
                    return

        watcher = threading.Thread(target=watch, daemon=True) if self.target is not None else None
        ctx.set_cancel_flag(flag)
        if watcher:
            watcher.start()
        try:
            film = scene.render(desc)
        except LiarGpuError as err:
            if err.code == LIAR_ERR_CANCELLED:
                return None
            raise
        finally:
            done.set()
            if watcher:
                watcher.join()
            ctx.set_cancel_flag(None)
        xyza, var = R.resolve(film)
        self.film = film
        if self.target is not None:
            self.target.write(xyza.astype(np.float32), var.astype(np.float32))
        return xyza
