"""RenderEngine of the scene API (src/liar/kernel/render_engine.cpp:170-358).

``engine.render()`` flattens ``engine.scene`` (cached until the scene object changes), renders
``sampler.samplesPerPixel`` samples of every pixel of ``sampler.resolution`` on the GPU with
``engine.tracer`` and hands the resolved XYZ + alpha film to ``engine.target``.
"""
from __future__ import annotations

import numpy as np

from . import render as R
from .trace import Context

_CTX: Context | None = None


def default_context() -> Context:
    global _CTX
    if _CTX is None:
        _CTX = Context(0)
    return _CTX


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
        w, h = self.sampler.resolution
        from .output import film_settings
        desc = R.render_desc(self.camera, w, h, self.sampler.samplesPerPixel, self.tracer,
                             seed=self.seed or getattr(self.sampler, "seed_", 0), **film_settings(self.target))
        film = self._scene().render(desc)
        xyza, var = R.resolve(film)
        self.film = film
        if self.target is not None:
            self.target.write(xyza.astype(np.float32), var.astype(np.float32))
        return xyza
