"""Batched rendering: many scenes / resolutions / sample counts in one CUDA-graph launch
(liar_gpu_batch_*, include/liar_gpu.h), and the autotuner that picks its launch shapes.

No reference counterpart: the reference renders one scene per RenderEngine.render() call
(src/liar/kernel/render_engine.cpp:170). Films live on the device (torch tensors, W x H x 8 sums).
"""
from __future__ import annotations

import ctypes as C
import json
import os
import time
from pathlib import Path

import numpy as np

from . import _native as N
from .render import CRenderDesc


class BatchItem(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("render", CRenderDesc), ("d_film", C.c_void_p)]


class BatchConfig(C.Structure):
    _fields_ = [("hero_wavelengths", C.c_int32), ("max_bounces", C.c_int32), ("wave_paths", C.c_int32),
                ("shade_blocks_per_sm", C.c_int32), ("trace", N.TraceConfig)]


def make_config(hero: int = 4, max_bounces: int = 0, wave_paths: int = 0, shade_blocks_per_sm: int = 0,
                trace: tuple[int, int] | None = None) -> BatchConfig:
    c = BatchConfig()
    c.hero_wavelengths = int(hero)
    c.max_bounces = int(max_bounces)
    c.wave_paths = int(wave_paths)
    c.shade_blocks_per_sm = int(shade_blocks_per_sm)
    if trace:
        c.trace.block_size, c.trace.smem_stack = int(trace[0]), int(trace[1])
    return c


class BatchRenderer:
    """entries: list of (GpuScene, CRenderDesc). Allocates one device film per entry."""

    def __init__(self, ctx, entries, config: BatchConfig | None = None):
        import torch
        self.ctx = ctx
        lib = ctx._lib
        dev = f"cuda:{ctx.device}"
        self.films = [torch.zeros((d.height, d.width, 8), dtype=torch.float32, device=dev) for _, d in entries]
        self.entries = entries
        items = (BatchItem * len(entries))()
        for k, ((gs, d), film) in enumerate(zip(entries, self.films)):
            items[k].scene = gs.handle.value if isinstance(gs.handle, C.c_void_p) else gs.handle
            items[k].render = d
            items[k].d_film = film.data_ptr()
        self.config = config or make_config()
        h = C.c_void_p()
        ctx.check(lib.liar_gpu_batch_create(ctx.handle, items, len(entries), C.byref(self.config), C.byref(h)))
        self.handle = h
        self.paths = int(sum(d.width * d.height * d.spp for _, d in entries))

    def reset_films(self):
        for f in self.films:
            f.zero_()

    def launch(self, stream: int | None = None) -> None:
        self.ctx.check(self.ctx._lib.liar_gpu_batch_launch(self.ctx.handle, self.handle, C.c_void_p(stream or 0)))

    def stats(self) -> dict:
        out = (C.c_ulonglong * 4)()
        self.ctx.check(self.ctx._lib.liar_gpu_batch_stats(self.handle, out))
        return {"paths": out[0], "segments": out[1], "hits": out[2], "waves": out[3]}

    def close(self):
        if getattr(self, "handle", None):
            self.ctx._lib.liar_gpu_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- autotuner


TRACE_SHAPES = [(128, 8), (128, 16), (128, 24), (256, 8), (256, 16)]
WAVE_SIZES = [1 << 20, 1 << 21, 1 << 22, 1 << 23]
SHADE_GRIDS = [8, 16]


def _signature(entries, hero: int) -> str:
    tris = sum(int(gs.flat.triangles.shape[0]) for gs, _ in entries)
    paths = sum(d.width * d.height * d.spp for _, d in entries)
    return f"items={len(entries)};tris~{tris >> 16};paths~{paths >> 20};hero={hero}"


def default_cache_path() -> Path:
    return Path(os.environ.get("LIAR_TUNE_CACHE", Path.home() / ".cache" / "liar_b200" / "batch_tune.json"))


def tune_batch(ctx, entries, hero: int = 4, cache: Path | None = None, probe_spp: int = 4, stream=None,
               trace_shapes=None, wave_sizes=None, shade_grids=None, log=None) -> tuple[BatchConfig, dict]:
    """Times the batch on a probe (the same items at probe_spp samples) for every candidate
    launch shape -- trace block x shared stack, wave size, shade grid -- coordinate by coordinate,
    and returns the fastest. Results are cached in a JSON file keyed by GPU and workload."""
    import torch
    cache = cache or default_cache_path()
    key = f"{torch.cuda.get_device_name(ctx.device)}|{_signature(entries, hero)}"
    try:
        table = json.loads(cache.read_text())
    except Exception:
        table = {}
    if key in table:
        c = table[key]
        return make_config(hero, 0, c["wave_paths"], c["shade_blocks_per_sm"], tuple(c["trace"])), {"cached": True, **c}
    probe = []
    for gs, d in entries:
        p = CRenderDesc.from_buffer_copy(d)
        p.spp = min(d.spp, probe_spp)
        probe.append((gs, p))
    best = {"trace": (128, 16), "wave_paths": 1 << 22, "shade_blocks_per_sm": 16}
    timings = []

    def time_cfg(cfg_dict):
        cfg = make_config(hero, 0, cfg_dict["wave_paths"], cfg_dict["shade_blocks_per_sm"], cfg_dict["trace"])
        br = BatchRenderer(ctx, probe, cfg)
        br.launch(stream)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(2):
            br.launch(stream)
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / 2
        br.close()
        timings.append({**{k: (list(v) if isinstance(v, tuple) else v) for k, v in cfg_dict.items()}, "s": dt})
        if log:
            log(f"tune {cfg_dict}: {dt * 1e3:.2f} ms")
        return dt

    best_t = time_cfg(best)
    for name, values in (("trace", trace_shapes or TRACE_SHAPES), ("wave_paths", wave_sizes or WAVE_SIZES),
                         ("shade_blocks_per_sm", shade_grids or SHADE_GRIDS)):
        for v in values:
            if v == best[name]:
                continue
            cand = dict(best)
            cand[name] = v
            t = time_cfg(cand)
            if t < best_t:
                best, best_t = cand, t
    rec = {"trace": list(best["trace"]), "wave_paths": best["wave_paths"],
           "shade_blocks_per_sm": best["shade_blocks_per_sm"], "probe_s": best_t}
    table[key] = rec
    try:
        cache.parent.mkdir(parents=True, exist_ok=True)
        cache.write_text(json.dumps(table, indent=1))
    except OSError:
        pass
    return make_config(hero, 0, best["wave_paths"], best["shade_blocks_per_sm"], best["trace"]), \
        {"cached": False, **rec, "candidates": timings}
