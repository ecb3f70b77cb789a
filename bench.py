#!/usr/bin/env python
"""Benchmark of the QBVH closest-hit path: 1,310,720-triangle displaced icosphere, 16,777,216
random rays (origins uniform in 1.5x the bounding box, directions uniform on the sphere).

One step = one closest-hit launch over all rays, rays already resident in HBM (``value``).
``e2e`` traces the same rays through the public C ABI entry point ``liar_gpu_trace`` from
pinned host buffers, copies in and out included. ``--impl reference`` times the CPU
restatement of the reference's path (oracle/) on the host cores instead.

Multi-GPU (torchrun): rays are independent, so each rank traces its own ray set against its own
replica of the mesh (weak scaling, no collective on the data path); rank 0 reports the total
rays of all ranks over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "QBVH closest-hit Mrays/s"
WORKLOAD = "displaced icosphere 1,310,720 tris, 16,777,216 random rays, closest hit"
LEVELS = 8
N_RAYS = 1 << 24


def load_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d.get("bf16_tflops", 1590.0)),
                "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


class ClockSampler:
    """Samples SM clocks and throttle reasons every 100 ms (one nvidia-smi -lms process) while
    the timed regions run."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            time.sleep(0.3)  # let the first sample land before the timed work starts
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self) -> dict:
        rows = [[x.strip() for x in ln.split(",")] for ln in self.lines]
        rows = [r for r in rows if len(r) >= 7]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[0]) for r in rows if num(r[0]) is not None]
        mx = [num(r[1]) for r in rows if num(r[1]) is not None]
        pw = [num(r[2]) for r in rows if num(r[2]) is not None]
        reasons = sorted({self.NAMES[k] for r in rows for k in range(4) if r[3 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(pw) if pw else None, "reasons": reasons, "samples": len(rows)}


def ctx_sms(ctx) -> int:
    import torch
    return torch.cuda.get_device_properties(ctx.device).multi_processor_count


def workload_config(world: int, n_triangles: int) -> dict:
    """The traversal workload's config, identical in both arms."""
    return {"workload": WORKLOAD, "triangles": int(n_triangles), "rays_per_step": N_RAYS,
            "parallelism": f"replicas{world}" if world > 1 else "single",
            "l2": "rays (512 MiB) stream through; larger than L2, no flush"}


def l2_read_peak(stream, device: str, sms: int) -> dict:
    """L2 read bandwidth of this GPU, measured by the project's probe kernel
    (liar_b200/probe/l2_read.cu): buffers of 16-64 MiB (inside the 126 MB L2) read 16 B at a time
    by 4 blocks of 512 threads per SM, many passes per launch; the best size's GB/s."""
    import ctypes as C
    import torch
    from liar_b200 import build
    lib = C.CDLL(str(build.PROBE_LIB))
    lib.liar_probe_l2_read.restype = C.c_int
    lib.liar_probe_l2_read.argtypes = [C.c_void_p, C.c_uint64, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    blocks = 4 * sms
    sink = torch.empty(blocks * 512, dtype=torch.int32, device=device)
    best, rows = 0.0, []
    for mib in (16, 32, 48, 64):
        buf = torch.randint(0, 1 << 30, (mib << 18,), dtype=torch.int32, device=device)  # mib MiB
        n_vec = buf.numel() // 4
        passes = max(1, (4 << 30) // buf.numel() // 4)  # about 4 GiB read per launch
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

        def launch():
            rc = lib.liar_probe_l2_read(C.c_void_p(buf.data_ptr()), n_vec, passes, blocks, C.c_void_p(sink.data_ptr()),
                                        C.c_void_p(stream.cuda_stream))
            if rc:
                raise RuntimeError(f"L2 probe launch failed: CUDA error {rc}")

        for _ in range(3):
            launch()
        e0.record(stream)
        for _ in range(5):
            launch()
        e1.record(stream)
        stream.synchronize()
        gbs = 5 * passes * buf.numel() * 4 / (e0.elapsed_time(e1) * 1e-3) / 1e9
        rows.append([mib, round(gbs, 1)])
        best = max(best, gbs)
        del buf
    return {"gbs": best, "by_buffer_mib": rows, "source": "measured (liar_b200/probe/l2_read.cu)"}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def replica_seed(rank: int) -> int:
    """Replicas trace their own ray sets: rank k draws the workload's rays with seed k."""
    return rank


def max_over_ranks(ms: float, world: int, dist, device) -> float:
    """A timed region's duration as the slowest rank saw it (one all-reduce, MAX)."""
    if world <= 1:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, units_per_rank: int, ms: float) -> float:
    """Units of all ranks over the slowest rank's time, per second (weak scaling: fixed units per rank)."""
    return world * units_per_rank / (ms * 1e-3)


def cpu_baseline_rays(v, f, rays, target_seconds=10.0):
    """Times the oracle tree on a bounded sample of the workload's rays (about target_seconds of
    CPU work on all host threads); returns (Mrays/s, info)."""
    import oracle
    threads = oracle.hardware_threads()
    tree = oracle.Tree(v, f)
    n = min(len(rays), 1 << 18)
    t0 = time.perf_counter()
    tree.trace(rays[:n], threads=threads)
    dt = max(time.perf_counter() - t0, 1e-3)
    total = int(n * target_seconds / dt)
    done, t0 = 0, time.perf_counter()
    while done < total:
        m = min(len(rays), total - done)
        tree.trace(rays[:m], threads=threads)
        done += m
    dt2 = time.perf_counter() - t0
    return done / dt2 / 1e6, {"cores": threads, "sample": f"{done} rays of the workload distribution (first "
                                                        f"{min(len(rays), total)} rays, repeated), {dt2:.1f} s "
                                                        f"on {threads} host threads"}


def cornell_bench(ctx, stream, args, world, dist, local, cpu: bool) -> dict:
    """Plain spectral path tracing of the Cornell workload (256 x 256, 16 spp, RR from generation 3,
    depth cap 8): samples/s and path segments/s on the device, CPU restatement beside it."""
    import torch
    from liar_b200 import render as R, scenes_render
    W, H, SPP = 256, 256, 16
    e = scenes_render.cornell_engine(W, H, SPP)
    flat = R.flatten(e.scene)
    gs = R.GpuScene(ctx, flat)
    desc = R.render_desc(e.camera, W, H, SPP, e.tracer, seed=0)
    film = torch.zeros((H, W, 8), dtype=torch.float32, device=f"cuda:{local}")
    for _ in range(max(3, args.warmup)):
        gs.render_device(desc, film.data_ptr(), stream.cuda_stream)
    stream.synchronize()
    steps = max(1, min(args.steps, 20))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        gs.render_device(desc, film.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    stream.synchronize()
    ms = e0.elapsed_time(e1) / steps
    ms = max_over_ranks(ms, world, dist, f"cuda:{local}")
    st = gs.stats()
    peaks = load_peaks()
    seg_s = world * st["segments"] / (ms * 1e-3)
    # per path segment through HBM: the trace kernel reads the queued ray (32 B + 4 B path index)
    # and writes its hit (8 B); the shade kernel reads ray, index and hit, reads and writes the
    # 24 B path state, and appends the next ray (36 B): 172 B. The 36-triangle tree stays in L1/L2.
    seg_bytes = 36 + 8 + 44 + 48 + 36
    out = {"workload": "Cornell box 256x256, 16 spp, single wavelength, RR from generation 3, max depth 8",
           "ms_per_frame": ms, "samples_per_s": world * st["paths"] / (ms * 1e-3),
           "segments_per_s": seg_s, "segments_per_sample": st["segments"] / st["paths"],
           "roofline": {"bound": "hbm", "achieved": seg_bytes * seg_s / world / 1e9, "peak": peaks["hbm_gbs"],
                        "unit": "GB/s", "frac": seg_bytes * seg_s / world / 1e9 / peaks["hbm_gbs"], "traffic": None,
                        "model": f"{seg_bytes} B per path segment (queued ray, hit, path state, next ray)",
                        "note": "a 36-triangle scene: latency- and issue-bound, far below the memory roofline"},
           "note": "device time of liar_gpu_render_device per frame; each bounce is launched against the queue "
                   "length on the device, the host reads a length only after the next bounce is queued"}
    # the same frame with the DirectLighting tracer (16 light + 16 BSDF samples per camera vertex)
    from liar_b200 import tracers
    dl = tracers.DirectLighting()
    ddesc = R.render_desc(e.camera, W, H, SPP, dl, seed=0)
    for _ in range(2):
        gs.render_device(ddesc, film.data_ptr(), stream.cuda_stream)
    stream.synchronize()
    dsteps = max(1, min(args.steps, 10))
    e0.record(stream)
    for _ in range(dsteps):
        gs.render_device(ddesc, film.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    stream.synchronize()
    dms = e0.elapsed_time(e1) / dsteps
    dms = max_over_ranks(dms, world, dist, f"cuda:{local}")
    out["direct_lighting"] = {"ms_per_frame": dms, "samples_per_s": world * W * H * SPP / (dms * 1e-3),
                              "shadow_rays_per_sample": 32,
                              "shadow_rays_per_s": world * W * H * SPP * 32 / (dms * 1e-3)}
    if cpu:
        import oracle
        rs = oracle.RenderScene(flat)

        def cpu_rate(d, seconds=2.0):
            """Whole frames (then rows, wrapping around) of d on all host threads for at least
            `seconds` of wall time; returns (samples/s, samples, s)."""
            cfilm = np.zeros((H, W, 8), np.float32)
            done, row, t0 = 0, 0, time.perf_counter()
            while time.perf_counter() - t0 < seconds:
                rows = min(16, H - row)
                rs.render(d, cfilm, pixels=(row * W, (row + rows) * W))
                done += rows * W * SPP
                row = (row + rows) % H
            dt = time.perf_counter() - t0
            return done / dt, done, dt

        val, n, dt = cpu_rate(desc)
        out["cpu_baseline"] = {"value": val, "unit": "samples/s", "cores": oracle.hardware_threads(), "kind": "port",
                               "sample": f"{n} samples ({n // (W * SPP)} image rows of 16 spp), {dt:.1f} s"}
        val, n, dt = cpu_rate(ddesc)
        out["direct_lighting"]["cpu_baseline"] = {
            "value": val, "unit": "samples/s", "cores": oracle.hardware_threads(), "kind": "port",
            "sample": f"{n} samples ({n // (W * SPP)} image rows of 16 spp) with DirectLighting, {dt:.1f} s"}
    gs.close()
    return out


def batch_bench(ctx, stream, args, world, dist, local, cpu: bool, n_scenes: int = 64) -> dict:
    """Batched rendering: 64 seeded procedural scenes (10k-2M triangles, 128^2-1024^2, 4-64 spp,
    log-uniform), 4 hero wavelengths, max depth 8, the whole batch as one CUDA-graph launch with
    launch shapes chosen by the autotuner. samples/s counts camera paths (each carries 4 wavelengths)."""
    import torch
    from liar_b200 import batch as B, render as R, scenes_batch as SB
    t0 = time.perf_counter()
    work = SB.batch_workload(n_scenes, seed=0)
    tracer = SB.batch_tracer()
    flats = [R.flatten(w.scene) for w in work]
    scenes = [R.GpuScene(ctx, f) for f in flats]
    entries = [(gs, R.render_desc(w.camera, w.width, w.height, w.spp, tracer, seed=k))
               for k, (gs, w) in enumerate(zip(scenes, work))]
    setup_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    cfg, tune = B.tune_batch(ctx, entries, hero=4, probe_spp=2, stream=stream.cuda_stream)
    tune_s = time.perf_counter() - t0
    br = B.BatchRenderer(ctx, entries, cfg)
    br.launch(stream.cuda_stream)                    # warm-up: the whole batch once
    stream.synchronize()
    steps = 2
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        br.launch(stream.cuda_stream)
    e1.record(stream)
    stream.synchronize()
    ms = e0.elapsed_time(e1) / steps
    ms = max_over_ranks(ms, world, dist, f"cuda:{local}")
    st = br.stats()
    peaks = load_peaks()
    seg_s = world * st["segments"] / (ms * 1e-3)
    # per path segment through HBM: trace reads the queued ray (36 B) and writes its hit (8 B);
    # shade reads ray and hit, reads and writes the path state of 4 hero wavelengths (16 + 12 x 4
    # = 64 B) and appends the next ray (36 B): 252 B; tree nodes and triangles are not counted
    seg_bytes = 36 + 8 + 44 + 128 + 36
    tris = [w.n_triangles for w in work]
    out = {"workload": f"{n_scenes} procedural scenes, {min(tris)}-{max(tris)} triangles ({sum(tris)} total), "
                       "128^2-1024^2, 4-64 spp, 4 hero wavelengths, RR from generation 3, max depth 8",
           "ms_per_batch": ms, "samples_per_s": world * st["paths"] / (ms * 1e-3),
           "segments_per_s": world * st["segments"] / (ms * 1e-3), "samples_per_batch": st["paths"],
           "segments_per_sample": st["segments"] / st["paths"], "waves": st["waves"],
           "graph_launches_per_batch": 1,
           "roofline": {"bound": "hbm", "achieved": seg_bytes * seg_s / world / 1e9, "peak": peaks["hbm_gbs"],
                        "unit": "GB/s", "frac": seg_bytes * seg_s / world / 1e9 / peaks["hbm_gbs"], "traffic": None,
                        "model": f"{seg_bytes} B per path segment (queued ray, hit, 4-wavelength path state, next "
                                 "ray); the trees' node and triangle reads are not counted, so this is a lower "
                                 "bound of the memory work"},
           "tuned": {"trace": [cfg.trace.block_size, cfg.trace.smem_stack],
                     "wave_paths": cfg.wave_paths, "shade_blocks_per_sm": cfg.shade_blocks_per_sm,
                     "cached": tune.get("cached", False), "seconds": tune_s},
           "setup_seconds": setup_s,
           "note": "device time of one cudaGraphLaunch per batch (WHILE node over waves, queue sizes on device)"}
    br.close()
    if cpu:
        import oracle
        # the CPU restatement (one wavelength per sample) on the middle rows of the smallest, the
        # median and the largest scene, about 4 s each
        order = np.argsort(tris)
        done, dt = 0, 0.0
        picked = []
        for k in (int(order[0]), int(order[len(order) // 2]), int(order[-1])):
            w, d = work[k], entries[k][1]
            rs = oracle.RenderScene(flats[k])
            film = np.zeros((d.height, d.width, 8), np.float32)
            row, t_scene = d.height // 2, 0.0
            while t_scene < 4.0 and row < d.height:
                rows = min(4, d.height - row)
                t1 = time.perf_counter()
                rs.render(d, film, pixels=(row * d.width, (row + rows) * d.width))
                t_scene += time.perf_counter() - t1
                done += rows * d.width * d.spp
                row += rows
            dt += t_scene
            picked.append(f"scene {k} ({w.n_triangles} tris, {w.width}^2, {w.spp} spp)")
        out["cpu_baseline"] = {"value": done / dt, "unit": "samples/s", "cores": oracle.hardware_threads(),
                               "kind": "port", "sample": f"{done} samples of {', '.join(picked)}, one wavelength "
                                                         f"per sample, {dt:.1f} s"}
    for gs in scenes:
        gs.close()
    return out


def guided_bench(ctx, stream, args, world, dist, local, cpu: bool, plain_curve: bool = False) -> dict:
    """Learned path guiding on the slit room (200k clutter triangles, 1024^2): time for guided
    rendering (online training included) to reach the error of a plain 1024-spp render, against a
    plain reference at args.guided_ref_spp (the reference's own variance is subtracted from each MSE).
    Also the guide network's tensor-core throughput (inference and one training step).
    plain_curve: also render the plain tracer in 16-spp chunks up to 1024 spp (outside the timed
    plain render) and record its MSE after every power-of-two spp, the plain half of the MSE-vs-time
    comparison."""
    import torch
    from liar_b200 import guiding as GD, render as R, scenes_guiding as SG
    res, ref_spp, plain_spp, chunk = args.guided_res, args.guided_ref_spp, 1024, 16
    dev = f"cuda:{local}"
    scene, cam = SG.slit_room(200_000)
    flat = R.flatten(scene)
    gs = R.GpuScene(ctx, flat)
    tracer = SG.guiding_tracer()
    st = stream.cuda_stream

    def film():
        return torch.zeros((res, res, 8), dtype=torch.float32, device=dev)

    def resolve(f):
        n = f[..., 7:8].clamp(min=1.0)
        mean = f[..., 0:3] / n
        var = (f[..., 4:7] / n - mean ** 2).clamp(min=0.0) / (n - 1).clamp(min=1.0)
        return mean, var

    ref = film()
    t0 = time.perf_counter()
    for k in range(0, ref_spp, 256):
        gs.render_device(R.render_desc(cam, res, res, min(256, ref_spp - k), tracer, seed=1_000_000, first_sample=k),
                         ref.data_ptr(), st)
    stream.synchronize()
    ref_s = time.perf_counter() - t0
    ref_mean, ref_var = resolve(ref)
    ref_var_term = float(ref_var.mean())

    def mse(f):
        m, _ = resolve(f)
        return float(((m - ref_mean) ** 2).mean()) - ref_var_term

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    plain = film()
    gs.render_device(R.render_desc(cam, res, res, 16, tracer, seed=5), film().data_ptr(), st)  # warm-up
    e0.record(stream)
    gs.render_device(R.render_desc(cam, res, res, plain_spp, tracer, seed=7), plain.data_ptr(), st)
    e1.record(stream)
    stream.synchronize()
    plain_s = e0.elapsed_time(e1) * 1e-3
    plain_mse = mse(plain)
    plain_stats = gs.stats()
    pcurve = []
    if plain_curve:
        pf, t_cum, spp = film(), 0.0, 0
        while spp < plain_spp:
            e0.record(stream)
            gs.render_device(R.render_desc(cam, res, res, chunk, tracer, seed=9, first_sample=spp), pf.data_ptr(), st)
            e1.record(stream)
            stream.synchronize()
            t_cum += e0.elapsed_time(e1) * 1e-3
            spp += chunk
            if spp & (spp - 1) == 0:
                pcurve.append((round(t_cum, 4), spp, mse(pf)))
        del pf
    # guided: chunks of 16 spp; during the first train_chunks chunks the guide trains after every
    # pass over the image (4 Adam steps of 16,384 records)
    c_guide, lp_guide, train_chunks = 0.4, 0.1, 4
    g = GD.Guide(ctx, GD.scene_bounds(flat), guide_probability=c_guide, light_probability=lp_guide,
                 learning_rate=5e-3, steps_per_pass=4, batch_records=16384, seed=0)
    gf = film()
    curve, t_cum, spp, t_hit = [], 0.0, 0, None
    while spp < 4 * plain_spp:
        d = R.render_desc(cam, res, res, chunk, tracer, seed=11, first_sample=spp)
        e0.record(stream)
        training = spp < train_chunks * chunk
        if training:
            d.wave_paths = res * res  # one training round per pass over the image
        g.render(gs, d, gf.data_ptr(), train=training, stream=st)
        e1.record(stream)
        stream.synchronize()
        dt = e0.elapsed_time(e1) * 1e-3
        prev_t, prev_m = t_cum, (curve[-1][2] if curve else None)
        t_cum += dt
        spp += chunk
        m = mse(gf)
        curve.append((round(t_cum, 4), spp, m))
        if m <= plain_mse and t_hit is None:
            # linear interpolation of the crossing inside the last chunk
            if prev_m is not None and prev_m > m:
                t_hit = prev_t + dt * (prev_m - plain_mse) / (prev_m - m)
            else:
                t_hit = t_cum
            break
    gstats = g.stats()
    # the network alone: inference over 1M vertices, one training step over 65,536 records
    x = torch.rand((1 << 20, 9), device=dev) * 2 - 1
    rec = torch.cat([torch.rand((65536, 9), device=dev) * 2 - 1, torch.nn.functional.normalize(
        torch.randn((65536, 3), device=dev), dim=1), torch.rand((65536, 1), device=dev)], 1).contiguous()
    g.eval(x, stream=st)
    g.train_step(rec, apply=True, stream=st)
    e0.record(stream)
    for _ in range(5):
        g.eval(x, stream=st)
    e1.record(stream)
    stream.synchronize()
    eval_s = e0.elapsed_time(e1) * 1e-3 / 5
    e0.record(stream)
    for _ in range(5):
        g.train_device(rec, apply=True, stream=st)
    e1.record(stream)
    stream.synchronize()
    train_s = e0.elapsed_time(e1) * 1e-3 / 5  # device time per step (CUDA events, no host waits)
    flop_fwd = 2 * (225 * 64 + 4 * 64 * 64 + 64 * 40)
    peaks = load_peaks()
    out = {"workload": f"slit room {res}x{res}, 200k box triangles, GGX floor, 6500 K light through a 0.2x2 slit; "
                       f"MLP 9 -> 225 (12 frequencies) -> 5x64 -> 8 vMF lobes, bf16",
           "reference_spp": ref_spp, "reference_seconds": ref_s,
           "plain": {"spp": plain_spp, "seconds": plain_s, "mse": plain_mse,
                     "samples_per_s": plain_spp * res * res / plain_s,
                     "segments_per_sample": plain_stats["segments"] / max(plain_stats["paths"], 1)},
           "guided": {"seconds_to_plain_mse": t_hit, "spp_at_crossing": spp if t_hit else None,
                      "training_chunks": train_chunks, "chunk_spp": chunk, "adam_steps": gstats["steps"],
                      "batch_records": 16384, "guide_probability": c_guide, "light_probability": lp_guide,
                      "curve_t_spp_mse": curve[:: max(1, len(curve) // 24)]},
           **({"plain_curve_t_spp_mse": pcurve} if plain_curve else {}),
           "time_ratio_guided_over_plain": (t_hit / plain_s) if t_hit else None,
           "network": {"inference_queries_per_s": (1 << 20) / eval_s,
                       "inference_tflops": flop_fwd * (1 << 20) / eval_s / 1e12,
                       "train_step_ms_65536": train_s * 1e3,
                       "train_tflops": 3 * flop_fwd * 65536 / train_s / 1e12,
                       "peak_bf16_tflops": peaks["bf16_tflops"],
                       "inference_frac_of_peak": flop_fwd * (1 << 20) / eval_s / 1e12 / peaks["bf16_tflops"]},
           "note": "MSE over XYZ against the plain reference, reference variance subtracted; guided time includes "
                   f"online training ({train_chunks} chunks x {chunk} passes x 4 Adam steps x 16,384 records)"}
    if cpu:
        import oracle
        rs = oracle.RenderScene(flat)
        cres = 256
        d = R.render_desc(cam, cres, cres, 16, tracer, seed=3)
        cfilm = np.zeros((cres, cres, 8), np.float32)
        rows, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < 2.0:  # whole 16-spp frames, repeated, for at least 2 s
            r0 = rows % cres
            rs.render(d, cfilm, pixels=(r0 * cres, (r0 + 4) * cres))
            rows += 4
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": rows * cres * 16 / dt, "unit": "samples/s", "cores": oracle.hardware_threads(),
                               "kind": "port", "sample": f"plain path tracing, {rows} rows (in passes over a {cres}^2 "
                                                         f"16-spp render) of the slit room, {dt:.1f} s"}
    g.close()
    gs.close()
    return out


def camera_queries(flat, cam, width, height):
    """Gather points of the photon workload: the first hits of the camera's pixel-centre rays on
    surfaces with a diffuse (Lambert) BSDF, with their normals flipped toward the camera."""
    from liar_b200 import render as R
    from liar_b200.trace import Mesh
    from liar_b200.kernel import default_context
    c = cam.flatten()
    ys, xs = np.mgrid[0:height, 0:width]
    sx, sy = (xs + 0.5) / width - 0.5, (ys + 0.5) / height - 0.5
    d = (np.asarray(c["direction"])[None, None] + sx[..., None] * np.asarray(c["right"])
         + sy[..., None] * np.asarray(c["down"])).reshape(-1, 3)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    o = np.broadcast_to(np.asarray(c["position"]), d.shape)
    rays = np.concatenate([o, np.full((len(d), 1), 1e-6), d, np.full((len(d), 1), np.inf)], axis=1).astype(np.float32)
    mesh = Mesh(default_context(), flat.vertices, flat.triangles)
    prim, t = mesh.intersect(rays)
    mesh.close()
    hit = prim >= 0
    mats = flat.object_material[flat.triangle_object[np.maximum(prim, 0)]]
    lam = np.array([m.type == R.MAT_LAMBERT for m in flat.materials])[np.maximum(mats, 0)] & (mats >= 0)
    ok = hit & lam
    pts = (o[ok] + t[ok, None] * d[ok]).astype(np.float32)
    tri = flat.vertices[flat.triangles[prim[ok]]].astype(np.float64)
    n = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    n = np.where((n * d[ok]).sum(axis=1, keepdims=True) > 0, -n, n).astype(np.float32)
    return np.ascontiguousarray(pts), np.ascontiguousarray(n)


def photon_bench(ctx, stream, args, world, dist, local, cpu: bool, n_photons: int = 10_000_000) -> dict:
    """Photon mapping workload: 10M photons in the global map, 1920 x 1080 gather points, k = 64."""
    import ctypes as C
    import torch
    from liar_b200 import photons, render as R, scenes_render
    K = 64
    scene, cam = scenes_render.photon_scene()
    flat = R.flatten(scene)
    gs = R.GpuScene(ctx, flat)
    desc = photons.photon_desc(n_photons, max_emitted=(1 << 32) - 1, ray_traced_direct=False, wave=1 << 22)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ph, counts = photons.trace_photons(gs, desc, capacity=n_photons + (3 << 22), stream=stream.cuda_stream)
    torch.cuda.synchronize()
    trace_s = time.perf_counter() - t0
    glob = (ph["tag"] & photons.GLOBAL) != 0
    pos = ph["position"][glob][:n_photons].contiguous()
    power = ph["power"][glob][:n_photons].contiguous()
    omega = ph["omega_in"][glob][:n_photons].contiguous()
    n_map = pos.shape[0]
    r = photons.automatic_radius(power.cpu().numpy(), counts["emitted"], K)
    q, qn = camera_queries(flat, cam, 1920, 1080)
    nq = q.shape[0]
    dq = torch.from_numpy(q).to(f"cuda:{local}")
    dqn = torch.from_numpy(qn).to(f"cuda:{local}")
    didx = torch.empty((nq, K), dtype=torch.int32, device=f"cuda:{local}")
    dd2 = torch.empty((nq, K), dtype=torch.float32, device=f"cuda:{local}")
    dcnt = torch.empty(nq, dtype=torch.int32, device=f"cuda:{local}")
    dest = torch.empty((nq, 3), dtype=torch.float32, device=f"cuda:{local}")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    pmap = photons.PhotonMap(ctx, device_ptr=pos.data_ptr(), n=n_map, r_max=r, stream=stream.cuda_stream)
    e1.record(stream)
    stream.synchronize()
    first_build_ms = e0.elapsed_time(e1)  # includes the first allocation of the map's buffers
    build_ms = 0.0
    for _ in range(3):  # rebuilds in the map's own buffers, as a render after the first one does
        e0.record(stream)
        pmap.rebuild(pos.data_ptr(), n_map, r, stream=stream.cuda_stream)
        e1.record(stream)
        stream.synchronize()
        build_ms += e0.elapsed_time(e1) / 3
    lib = ctx._lib

    def gather():
        pmap.gather_device(dq.data_ptr(), nq, K, didx.data_ptr(), dd2.data_ptr(), dcnt.data_ptr(), stream.cuda_stream)

    def estimate():
        ctx.check(lib.liar_gpu_photon_estimate_device(
            ctx.handle, C.c_void_p(power.data_ptr()), C.c_void_p(omega.data_ptr()), n_map, C.c_void_p(dqn.data_ptr()),
            nq, K, C.c_void_p(didx.data_ptr()), C.c_void_p(dd2.data_ptr()), C.c_void_p(dcnt.data_ptr()),
            C.c_float(1.0 / counts["emitted"]), C.c_void_p(dest.data_ptr()), C.c_void_p(stream.cuda_stream)))

    for _ in range(max(3, args.warmup)):
        gather()
        estimate()
    stream.synchronize()
    steps = max(1, min(args.steps, 20))
    e0.record(stream)
    for _ in range(steps):
        gather()
    e1.record(stream)
    stream.synchronize()
    g_ms = e0.elapsed_time(e1) / steps
    e0.record(stream)
    for _ in range(steps):
        estimate()
    e1.record(stream)
    stream.synchronize()
    est_ms = e0.elapsed_time(e1) / steps
    ctx.synchronize()
    found = dcnt.float().mean().item()
    # algorithmic bytes per query: 12 B point + k x 36 B photon records (the reference's Photon) +
    # 27 x 8 B bucket ranges + k x 8 B results + 4 B count
    bytes_q = 12 + K * 36 + 27 * 8 + K * 8 + 4
    peaks = load_peaks()
    gbs = bytes_q * nq / (g_ms * 1e-3) / 1e9
    out = {"workload": "glass sphere + GGX copper panel + Lambert ground, 5000 K point light; "
                       f"{n_map} global photons, 1920x1080 gather points ({nq} on diffuse surfaces), k = {K}",
           "photons_emitted": counts["emitted"], "photon_trace_s": trace_s,
           "photons_stored_per_s": counts["stored"] / trace_s, "estimation_radius": r, "map_build_ms": build_ms, "first_map_build_ms": first_build_ms,
           "gather_ms": g_ms, "queries_per_s": world * nq / (g_ms * 1e-3), "mean_neighbours": found,
           "gather_gbs_algorithmic": gbs, "estimate_ms": est_ms,
           "roofline": {"bound": "hbm", "achieved": gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                        "frac": gbs / peaks["hbm_gbs"], "traffic": None,
                        "model": f"{bytes_q} B per query: 12 B point, {K} x 36 B photon records, 27 x 8 B bucket "
                                 f"ranges, {K} x 8 B results, 4 B count",
                        "kernel": "k_gather"}}
    if cpu:
        import oracle
        ns = min(nq, 20000)
        sel = np.random.default_rng(0).choice(nq, ns, replace=False)
        P = pos.cpu().numpy()
        t0 = time.perf_counter()
        oracle.knn_grid(P, q[sel[:1]], K, r)  # the grid build alone
        t_build = time.perf_counter() - t0
        t0 = time.perf_counter()
        ci, cd, cc = oracle.knn_grid(P, q[sel], K, r)
        dt = max(time.perf_counter() - t0 - t_build, 1e-6)
        out["cpu_baseline"] = {"value": ns / dt, "unit": "queries/s", "cores": oracle.hardware_threads(),
                               "kind": "port", "sample": f"{ns} of the {nq} gather points (grid k-NN), {dt:.2f} s "
                                                        f"after a {t_build:.1f} s grid build"}
        out["parity_sample"] = {"queries": ns, "identical_neighbour_sets":
                                bool((didx.cpu().numpy()[sel] == ci).all() and (dcnt.cpu().numpy()[sel] == cc).all())}
    pmap.close()
    # the PhotonMapper tracer end to end on the same scene: a global map of n_photons photons
    # (direct light from the map, as the gather workload above; k = 64 for both maps), then
    # 1920 x 1080 at 1 sample per pixel; the maps are built by the first render and kept
    from liar_b200 import tracers
    pm = tracers.PhotonMapper()
    pm.maxRayGeneration = 8
    pm.globalMapSize = n_photons
    pm.isRayTracingDirect = False
    pm.setEstimationSize("global", K)
    pm.setEstimationSize("caustic", K)
    film = torch.zeros((1080, 1920, 8), dtype=torch.float32, device=f"cuda:{local}")
    t0 = time.perf_counter()
    gs.render_device(R.render_desc(cam, 1920, 1080, 1, pm, seed=0), film.data_ptr(), stream.cuda_stream)
    stream.synchronize()
    first_s = time.perf_counter() - t0
    st = R.photon_mapper_stats(ctx)
    gs.render_device(R.render_desc(cam, 1920, 1080, 1, pm, seed=0, first_sample=1), film.data_ptr(), stream.cuda_stream)
    e0.record(stream)
    for k in range(2):
        gs.render_device(R.render_desc(cam, 1920, 1080, 1, pm, seed=0, first_sample=2 + k), film.data_ptr(),
                         stream.cuda_stream)
    e1.record(stream)
    stream.synchronize()
    frame_ms = e0.elapsed_time(e1) / 2
    out["photon_mapper_render"] = {
        "workload": f"PhotonMapper 1920x1080, 1 spp, global map {st['global']} photons, caustic map "
                    f"{st['caustic']}, k = {K}, direct light from the global map, max generation 8",
        "photons_shot": st["emitted"], "radii": st["radius"], "first_render_with_map_build_s": first_s,
        "frame_ms": frame_ms, "samples_per_s": 1920 * 1080 / (frame_ms * 1e-3)}
    del film
    gs.close()
    # the reference's classic photon-mapping example (examples/cornell_box/photon_mapper_classic.py):
    # the Cornell box, 200,000 global photons, 36 final gather rays over the precomputed irradiance
    # map (ratio 0.25), traced direct light, 800 x 800 x 4 spp
    scene, cam = scenes_render.cornell_box()
    gs = R.GpuScene(ctx, R.flatten(scene))
    pm = tracers.PhotonMapper()
    pm.maxNumberOfPhotons = 10_000_000
    pm.globalMapSize = 200_000
    pm.numFinalGatherRays = 36
    pm.ratioPrecomputedIrradiance = 0.25
    film = torch.zeros((800, 800, 8), dtype=torch.float32, device=f"cuda:{local}")
    t0 = time.perf_counter()
    gs.render_device(R.render_desc(cam, 800, 800, 1, pm, seed=0), film.data_ptr(), stream.cuda_stream)
    stream.synchronize()
    first_s = time.perf_counter() - t0
    st = R.photon_mapper_stats(ctx)
    e0.record(stream)
    gs.render_device(R.render_desc(cam, 800, 800, 4, pm, seed=0, first_sample=1), film.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    stream.synchronize()
    frame_ms = e0.elapsed_time(e1)
    out["photon_mapper_classic"] = {
        "workload": f"Cornell box, PhotonMapper with 36 final gather rays, global map {st['global']} photons, "
                    f"caustic map {st['caustic']}, irradiance ratio 0.25, 800x800 x 4 spp",
        "photons_shot": st["emitted"], "first_render_with_maps_s": first_s, "frame_ms": frame_ms,
        "samples_per_s": 800 * 800 * 4 / (frame_ms * 1e-3),
        "gather_rays_per_s": 800 * 800 * 4 * 36 / (frame_ms * 1e-3)}
    del film
    gs.close()
    return out


def run_reference(args, world, rank):
    """The reference arm: the CPU restatement of the reference's path (oracle/: the same 4-wide
    SAH tree restated on the host and the exact triangle test) on all host threads, tracing all
    16,777,216 workload rays per step, through the same timed-step structure as our arm."""
    if rank != 0:
        return
    import oracle
    from liar_b200 import scenes
    v, f = scenes.displaced_icosphere(LEVELS, seed=0)
    rays = scenes.random_rays(v, N_RAYS, seed=0)
    threads = oracle.hardware_threads()
    tree = oracle.Tree(v, f)
    for _ in range(args.warmup):
        tree.trace(rays, threads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        tree.trace(rays, threads=threads)
        times.append(time.perf_counter() - t0)
    dt = float(np.mean(times))
    val = N_RAYS / dt / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural mesh and rays)",
        "config": workload_config(world, f.shape[0]),
        "cpu_baseline": {"value": val, "unit": "Mrays/s", "cores": threads, "kind": "port",
                         "sample": f"all {N_RAYS} workload rays per step, closest hit (CPU restatement; the "
                                   f"reference's Lass core cannot be built)"},
        "e2e": {"value": val, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_case(name: str) -> None:
    """Small single-kernel workloads for profiling captures (ncu -k ... python bench.py --case NAME):
    guide-eval (the guide network over 1M random vertices, 3 launches), direct (DirectLighting on
    the Cornell frame, 256^2 x 4 spp, twice), shade (the Cornell path-tracing frame, twice),
    gather (k = 64 over 4M uniform photons for 256k uniform queries, twice), gather-photon (the
    photon workload's gather: 10M photons, the 1080p camera queries, k = 64, twice), guided (the slit
    room at 256^2: 4 training passes, then 16 guided samples per pixel), guided-crossing (the guiding
    workload against a 65,536-spp plain reference, both MSE curves), pm (the PhotonMapper on
    the photon scene, 1M global photons, 480 x 270, two frames)."""
    import torch
    from liar_b200.kernel import default_context
    ctx = default_context()
    if name == "guide-eval":
        from liar_b200 import guiding as GD
        g = GD.Guide(ctx, (np.array([-1, -1, -1], np.float32), np.array([1, 1, 1], np.float32)))
        x = torch.rand((1 << 20, 9), device="cuda", generator=torch.Generator("cuda").manual_seed(0)) * 2 - 1
        st = torch.cuda.Stream()  # a stream of its own: the events must see the network's kernels
        for _ in range(3):
            g.eval(x, stream=st.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        for _ in range(5):
            g.eval(x, stream=st.cuda_stream)
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 5
        flop = 2 * (225 * 64 + 4 * 64 * 64 + 64 * 40) * (1 << 20)
        print(json.dumps({"case": name, "eval_device_ms_1M": ms, "tflops": flop / (ms * 1e-3) / 1e12}))
    elif name == "guide-train":
        # twenty Adam steps over 65,536 random records, device-timed
        from liar_b200 import guiding as GD
        g = GD.Guide(ctx, (np.array([-1, -1, -1], np.float32), np.array([1, 1, 1], np.float32)))
        gen = torch.Generator("cuda").manual_seed(0)
        rec = torch.cat([torch.rand((65536, 9), device="cuda", generator=gen) * 2 - 1, torch.nn.functional.normalize(
            torch.randn((65536, 3), device="cuda", generator=gen), dim=1),
            torch.rand((65536, 1), device="cuda", generator=gen)], 1).contiguous()
        g.train_step(rec)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        st = torch.cuda.Stream()  # a stream of its own: the events must see the training kernels
        torch.cuda.synchronize()
        e0.record(st)
        for _ in range(20):
            g.train_device(rec, stream=st.cuda_stream)
        e1.record(st)
        torch.cuda.synchronize()
        print(json.dumps({"case": name, "train_step_device_ms": e0.elapsed_time(e1) / 20}))
    elif name in ("direct", "shade"):
        from liar_b200 import render as R, scenes_render, tracers
        e = scenes_render.cornell_engine(256, 256, 16)
        gs = R.GpuScene(ctx, R.flatten(e.scene))
        film = torch.zeros((256, 256, 8), device="cuda")
        d = (R.render_desc(e.camera, 256, 256, 4, tracers.DirectLighting()) if name == "direct"
             else R.render_desc(e.camera, 256, 256, 16, e.tracer))
        for _ in range(2):
            gs.render_device(d, film.data_ptr())
    elif name == "guided-crossing":
        # the guiding workload measured against its stated reference: a plain 65,536-spp render of
        # the slit room at 1024^2 (about 2.5 minutes), the plain MSE-vs-time curve beside the guided one
        stream = torch.cuda.Stream()
        args = argparse.Namespace(guided_res=1024, guided_ref_spp=65536)
        out = guided_bench(ctx, stream, args, 1, None, 0, cpu=False, plain_curve=True)
        print(json.dumps({"case": name, "guided": out}), flush=True)
    elif name == "guided":
        from liar_b200 import guiding as GD, render as R, scenes_guiding as SG
        scene, cam = SG.slit_room(200_000)
        flat = R.flatten(scene)
        gs = R.GpuScene(ctx, flat)
        g = GD.Guide(ctx, GD.scene_bounds(flat), guide_probability=0.7, light_probability=0.1, learning_rate=5e-3,
                     steps_per_pass=4, batch_records=16384, seed=0)
        film = torch.zeros((256, 256, 8), device="cuda")
        d = R.render_desc(cam, 256, 256, 4, SG.guiding_tracer(), seed=1)
        d.wave_paths = 256 * 256
        g.render(gs, d, film.data_ptr(), train=True)
        g.render(gs, R.render_desc(cam, 256, 256, 16, SG.guiding_tracer(), seed=2), film.data_ptr(), train=False)
    elif name == "pm":
        from liar_b200 import render as R, scenes_render, tracers
        scene, cam = scenes_render.photon_scene()
        gs = R.GpuScene(ctx, R.flatten(scene))
        t = tracers.PhotonMapper()
        t.globalMapSize = 1_000_000
        t.isRayTracingDirect = False
        t.setEstimationSize("global", 64)
        t.setEstimationSize("caustic", 64)
        film = torch.zeros((270, 480, 8), device="cuda")
        for k in range(2):
            gs.render_device(R.render_desc(cam, 480, 270, 1, t, seed=0, first_sample=k), film.data_ptr())
    elif name == "gather-photon":
        # the photon workload's gather: 10M global photons of the photon scene, the 1920 x 1080
        # camera queries on diffuse surfaces, k = 64, twice
        from liar_b200 import photons as PH, render as R, scenes_render
        scene, cam = scenes_render.photon_scene()
        flat = R.flatten(scene)
        gs = R.GpuScene(ctx, flat)
        desc = PH.photon_desc(10_000_000, max_emitted=(1 << 32) - 1, ray_traced_direct=False, wave=1 << 22)
        ph, counts = PH.trace_photons(gs, desc, capacity=10_000_000 + (3 << 22))
        glob = (ph["tag"] & PH.GLOBAL) != 0
        pos = ph["position"][glob][:10_000_000].contiguous()
        r = PH.automatic_radius(ph["power"][glob][:10_000_000].cpu().numpy(), counts["emitted"], 64)
        q, _ = camera_queries(flat, cam, 1920, 1080)
        m = PH.PhotonMap(ctx, device_ptr=pos.data_ptr(), n=pos.shape[0], r_max=r)
        dq = torch.from_numpy(q).cuda()
        nq = q.shape[0]
        di = torch.empty((nq, 64), dtype=torch.int32, device="cuda")
        dd = torch.empty((nq, 64), dtype=torch.float32, device="cuda")
        dc = torch.empty(nq, dtype=torch.int32, device="cuda")
        for _ in range(2):
            m.gather_device(dq.data_ptr(), nq, 64, di.data_ptr(), dd.data_ptr(), dc.data_ptr(), 0)
    elif name == "gather":
        from liar_b200 import photons as PH
        rng = np.random.default_rng(0)
        m = PH.PhotonMap(ctx, rng.random((1 << 22, 3)).astype(np.float32), 0.02)
        q = rng.random((1 << 18, 3)).astype(np.float32)
        for _ in range(2):
            m.gather(q, 64)
    else:
        raise SystemExit(f"unknown case {name}")
    torch.cuda.synchronize()
    print(json.dumps({"case": name, "ok": True}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-workloads", action="store_true", help="only the traversal workload")
    ap.add_argument("--batch-scenes", type=int, default=64, help="scenes in the batched-rendering workload")
    ap.add_argument("--only", default="", help="comma list of workloads to run (cornell,photon,batch,guided); default all")
    ap.add_argument("--guided-res", type=int, default=1024, help="image side of the guiding workload")
    ap.add_argument("--guided-ref-spp", type=int, default=4096, help="samples per pixel of its plain reference")
    ap.add_argument("--case", default="", help="run one small profiling workload instead (see run_case)")
    args = ap.parse_args()
    if args.case:
        return run_case(args.case)
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    world, rank, local = dist_setup()
    if args.impl == "reference":
        return run_reference(args, world, rank)

    import torch
    import torch.distributed as dist
    from liar_b200 import scenes
    from liar_b200.trace import Context, Mesh

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    v, f = scenes.displaced_icosphere(LEVELS, seed=0)
    rays = scenes.random_rays(v, N_RAYS, seed=replica_seed(rank))
    ctx = Context(local)
    mesh = Mesh(ctx, v, f)
    stats = mesh.stats
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    d_rays = torch.from_numpy(rays).to(f"cuda:{local}")
    d_hits = torch.empty((N_RAYS, 2), dtype=torch.int32, device=f"cuda:{local}")
    d_cnt = torch.zeros(2, dtype=torch.int64, device=f"cuda:{local}")
    torch.cuda.synchronize()

    # visit counts of this exact ray set (one counted launch, outside the timed region)
    with torch.cuda.stream(stream):
        mesh.trace_into(d_rays.data_ptr(), N_RAYS, d_hits.data_ptr(), stream=stream.cuda_stream,
                        counters_ptr=d_cnt.data_ptr())
    stream.synchronize()
    ctx.synchronize()
    nodes_visited, tris_tested = d_cnt.cpu().tolist()

    def step(any_hit=False):
        mesh.trace_into(d_rays.data_ptr(), N_RAYS, d_hits.data_ptr(), any_hit=any_hit, stream=stream.cuda_stream)

    d_rays_any = d_rays.clone()
    d_rays_any[:, 7] = 0.5

    def step_any():
        mesh.trace_into(d_rays_any.data_ptr(), N_RAYS, d_hits.data_ptr(), any_hit=True, stream=stream.cuda_stream)

    # end to end through the C ABI with pinned host buffers, copies included
    h_rays = torch.from_numpy(rays).pin_memory()
    h_hits = torch.empty((N_RAYS, 2), dtype=torch.int32).pin_memory()
    lib = ctx._lib
    import ctypes as C

    def e2e_step():
        ctx.check(lib.liar_gpu_trace(ctx.handle, mesh.handle, C.c_void_p(h_rays.data_ptr()), N_RAYS,
                                     C.c_void_p(h_hits.data_ptr()), 0))

    def timed(fn, steps):
        """Device time per step of fn on the trace stream (CUDA events, synchronised both sides)."""
        for _ in range(args.warmup):
            fn()
        stream.synchronize()
        ctx.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        stream.synchronize()
        ctx.synchronize()
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1) / steps, world, dist, f"cuda:{local}")

    e2e_steps = max(1, min(args.steps, 20))
    with ClockSampler(local) as clocks:
        ms = timed(step, args.steps)
        ms_any = timed(step_any, args.steps)
        e2e_s = timed(e2e_step, e2e_steps) * 1e-3
    del d_rays_any
    value = whole_job_rate(world, N_RAYS, ms) / 1e6
    e2e_val = whole_job_rate(world, N_RAYS, e2e_s * 1e3) / 1e6

    peaks = load_peaks()
    l2 = l2_read_peak(stream, f"cuda:{local}", ctx_sms(ctx))
    per_ray_model = 128.0 * nodes_visited / N_RAYS + 48.0 * tris_tested / N_RAYS + 40.0
    achieved = per_ray_model * N_RAYS / (ms * 1e-3) / 1e9
    traffic = None
    prof = ROOT / "profiles" / "trace_closest_traffic.json"
    if prof.exists():
        traffic = json.loads(prof.read_text()).get("dram_bytes_per_launch")

    line = {
        "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded procedural mesh and rays)",
        "config": workload_config(world, stats["n_triangles"]),
        "tree": {k: stats[k] for k in ("n_nodes", "n_leaves", "max_depth", "stack_needed", "sah_cost",
                                       "device_bytes", "build_seconds")},
        "any_hit": {"value": world * N_RAYS / (ms_any * 1e-3) / 1e6, "unit": "Mrays/s", "tmax": 0.5,
                    "ms_per_step": ms_any},
        "visits_per_ray": {"nodes": nodes_visited / N_RAYS, "triangles": tris_tested / N_RAYS},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                     "model": "128 B x nodes visited + 48 B x triangles tested + 40 B per ray, counted on device",
                     "peak_source": peaks["source"],
                     "l2": {"peak": l2["gbs"], "frac": achieved / l2["gbs"], "unit": "GB/s",
                            "peak_by_buffer_mib": l2["by_buffer_mib"], "peak_source": l2["source"]}},
        "e2e": {"value": e2e_val, "unit": "Mrays/s", "h2d_bytes_per_step": N_RAYS * 32,
                "d2h_bytes_per_step": N_RAYS * 8, "api": "liar_gpu_trace (host buffers, pinned)"},
        "gpu_launches": args.steps,
        "clocks": clocks.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        val, info = cpu_baseline_rays(v, f, rays)
        line["cpu_baseline"] = {"value": val, "unit": "Mrays/s", "cores": info["cores"], "kind": "port",
                                "sample": info["sample"]}
    mesh.close()
    if not args.no_workloads:
        cpu_leg = rank == 0 and world == 1 and not args.no_cpu_baseline
        only = set(filter(None, args.only.split(",")))
        if not only or "cornell" in only:
            line["cornell"] = cornell_bench(ctx, stream, args, world, dist, local, cpu=cpu_leg)
        if not only or "photon" in only:
            line["photon"] = photon_bench(ctx, stream, args, world, dist, local, cpu=cpu_leg)
        if not only or "guided" in only:
            line["guided"] = guided_bench(ctx, stream, args, world, dist, local, cpu=cpu_leg)
        if not only or "batch" in only:
            line["batch"] = batch_bench(ctx, stream, args, world, dist, local, cpu=cpu_leg, n_scenes=args.batch_scenes)
    ctx.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
