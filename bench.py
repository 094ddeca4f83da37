#!/usr/bin/env python
"""Throughput of the advection hot path on the B200, one JSON line.

Workload (the throughput configuration): a 256^3 FP32 curl-noise field
(sigma 4 cells, field seed 1, spacing 1, unit RMS speed), 1,048,576 seeds
uniform in the valid domain [0, 255)^3 (seed 1; rank r uses seed 1 + r),
runge_kutta_4 with the reference's semantics, step 0.25, 2000 iterations,
end positions only. One bench step advects every seed through all its
iterations: particle state reset on the device, processing order, advection.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

`value` is whole-job particle-steps/s (steps actually taken, summed over
ranks, divided by the max over ranks of the device-timed step). `e2e` is the
same metric through the host C ABI call (dpa_advect_round) with pinned host
buffers, copies included. The CPU baseline is the oracle's reference-faithful
restatement on a bounded seed sample on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
import types
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "RK4 particle-steps/s vs plain FP32 GPU & host TBB; served p50/p99 latency"
UNIT = "particle-steps/s"
FALLBACK_HBM_GBS = 6650.0
BYTES_PER_STEP = {"f32": 96, "f16": 48, "bf16": 48}  # 8 corners x 3 components
STATE_BYTES = 12 + 8 + 12 + 8 + 1  # positions + remaining in, out + termination


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=30)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="dpa_b200", choices=["dpa_b200", "reference"])
    p.add_argument("--workload", default="throughput", choices=["throughput", "ftle", "recording"],
                   help="throughput: the headline configuration (curl noise 256^3, 1M seeds x "
                        "2000 steps, end positions); ftle: ABC + noise 256^3, 128^3 lattice x "
                        "250 steps, then FTLE; recording: ABC 64^3, 4096 seeds x 1000 steps, "
                        "curves with uint32 indices")
    p.add_argument("--storage", default="f32", choices=["f32", "f16", "bf16"])
    p.add_argument("--integrator", default="runge_kutta_4")
    p.add_argument("--grid", dest="n", type=int, default=256,
                   help="grid points per axis of the throughput workload")
    p.add_argument("--seeds", type=int, default=1 << 20)
    p.add_argument("--iterations", type=int, default=2000)
    p.add_argument("--step-size", type=float, default=0.25)
    p.add_argument("--cpu-seconds", type=float, default=10.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-systems", action="store_true",
                   help="skip the batched / graph / serving measurements")
    p.add_argument("--serve-seconds", type=float, default=60.0,
                   help="seconds of Poisson arrivals in the serving measurement")
    p.add_argument("--batch-n", type=int, default=512)
    return p.parse_args()


def workload_config(a, world):
    return {
        "workload": f"curl-noise {a.n}^3 {a.storage.upper()} field (sigma 4, seed 1, spacing 1), "
                    f"{a.seeds} uniform seeds per rank (seed 1+rank) in [0,{a.n - 1})^3, "
                    f"{a.integrator} (one field sample per step), step {a.step_size}, "
                    f"{a.iterations} iterations, end positions only",
        "field_shape": [a.n, a.n, a.n],
        "seeds_per_rank": a.seeds,
        "iterations": a.iterations,
        "step_size": a.step_size,
        "integrator": a.integrator,
        "storage": a.storage,
        "parallelism": f"replicas x{world} (independent seed sets, no collective)",
        "l2": "256 MiB buffer written between timed steps (L2 flush)",
    }


def measured_peak_hbm():
    path = ROOT / "MEASURED_PEAKS.json"
    try:
        d = json.loads(path.read_text())
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback 6.65 TB/s (MEASURED_PEAKS.json absent)"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        sms, maxes, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sms.append(float(parts[1]))
                maxes.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sms:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sms), "sm_max_mhz": max(maxes),
                "reasons": sorted(reasons), "samples": len(sms)}


def rank_seeds(grid, count, iterations, rank):
    """The seed set of one replica: `count` uniform seeds in the valid domain
    of the grid, drawn from stream 1 + rank, so every rank advects its own
    independent particles through the same (replicated) field."""
    from dpa_b200 import seeds
    offset, size = seeds.seed_box(grid)
    box = ([0.0, 0.0, 0.0], [float(s - 1) for s in grid.shape])
    return seeds.generate_random(offset, size, count, iterations, aabb=box, seed=1 + rank)


def make_inputs(a, rank, device):
    from dpa_b200 import fields
    grid = fields.curl_noise(a.n, 4.0, 1, spacing=1.0, device=device)
    return grid, rank_seeds(grid, a.seeds, a.iterations, rank)


def combine_over_ranks(ms, steps, device):
    """Whole-job figures of the replicas: the slowest rank's time and the
    particle-steps of all ranks (max and sum over the process group when there
    is one). Returns (ms_max, steps_total)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    n = torch.tensor([float(steps)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(n, op=dist.ReduceOp.SUM)
    return float(t.item()), float(n.item())


def cpu_baseline(a, grid, parts, target_seconds, steps_budget=None):
    """The oracle's reference-faithful restatement on a seed sample sized for
    about `target_seconds` of work on all host threads."""
    from oracle import binding as ob
    ob.build()
    threads = os.cpu_count() or 1
    ob.set_threads(threads)
    og = ob.OracleGrid.of(grid)
    rem = np.full(a.seeds, a.iterations, np.uint64)
    calib = max(threads * 8, 64)
    t0 = time.perf_counter()
    r = ob.advect_round(og, a.integrator, a.step_size, parts.position[:calib], rem[:calib])
    dt = time.perf_counter() - t0
    rate = float(np.sum(r.steps)) / max(dt, 1e-9)
    steps_per_particle = max(float(np.mean(r.steps)), 1.0)
    count = int(min(a.seeds, max(calib, rate * target_seconds / steps_per_particle)))
    t0 = time.perf_counter()
    r = ob.advect_round(og, a.integrator, a.step_size, parts.position[:count], rem[:count])
    dt = time.perf_counter() - t0
    taken = float(np.sum(r.steps))
    return {"value": taken / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"first {count} of the {a.seeds} seeds at full {a.iterations} iterations "
                      f"({int(taken)} particle-steps in {dt:.2f} s; oracle/oracle.cpp, "
                      "OpenMP dynamic schedule standing in for TBB)"}


def fp64_error(a, ctx, field, grid, parts, sample=512, horizons=(50, 250, None), integrator=None):
    """Position error of the GPU path against the FP64 oracle integrator, in
    cells, over the first `sample` seeds that complete in both, at several
    horizons (the field is chaotic: FP32 and FP64 trajectories separate
    exponentially, so only short horizons measure the integrator)."""
    from dpa_b200 import ParticleAdvector, Particles
    from oracle import binding as ob
    ob.build()
    ob.set_threads(os.cpu_count() or 1)
    og = ob.OracleGrid.of(grid)
    out = {"sample": sample}
    integrator = integrator or a.integrator
    adv = ParticleAdvector(ctx, sample, "none", integrator, a.step_size, False, False)
    for h in horizons:
        h = a.iterations if h is None else min(h, a.iterations)
        gpu = adv.advect(field, Particles.create(parts.position[:sample], h)).inactive_particles
        ref = ob.advect64(og, integrator, a.step_size, parts.position[:sample],
                          np.full(sample, h, np.uint64))
        ok = (ref.termination == 0) & (gpu.termination == 0)
        err = np.linalg.norm(gpu.position[ok].astype(np.float64) - ref.positions[ok], axis=1)
        err = err / float(grid.spacing[0])
        out[f"steps_{h}"] = {
            "completed": int(ok.sum()),
            "median_cells": float(np.median(err)) if ok.any() else None,
            "max_cells": float(np.max(err)) if ok.any() else None,
            "within_1e-3_cells": float(np.mean(err <= 1e-3)) if ok.any() else None}
    return out


def precision_forms(a, ctx, grid, parts, p0, r0, pos, rem, term, stream, f32_kernel_ms,
                    steps=5):
    """The same workload with the field stored in FP16 and BF16 (FP32
    interpolation and accumulation): kernel time, speed-up over this run's
    FP32 kernel, and position error against the FP64 oracle."""
    import ctypes as C
    from dpa_b200 import _native as N
    lib = ctx._lib
    out = {}
    for storage in ("f16", "bf16"):
        if storage == a.storage:
            continue
        field = ctx.field(grid, storage)
        opts = N.AdvectOptions(N.INTEGRATORS[a.integrator], float(np.float32(a.step_size)),
                               0, 0, 0, 1)
        times = []
        for i in range(steps + 2):
            pos.copy_(p0)
            rem.copy_(r0)
            ctx.check(lib.dpa_advect_device(ctx.handle, field.handle, C.byref(opts), a.seeds,
                                            C.c_void_p(pos.data_ptr()), C.c_void_p(rem.data_ptr()),
                                            C.c_void_p(term.data_ptr()),
                                            C.c_void_p(stream.cuda_stream)))
            o, k = C.c_float(), C.c_float()
            ctx.check(lib.dpa_context_last_timing(ctx.handle, C.byref(o), C.byref(k)))
            if i >= 2:
                times.append(k.value)
        steps_taken = float((a.iterations - rem.cpu().numpy().astype(np.int64)).sum())
        kernel = statistics.mean(times)
        out[storage] = {"kernel_ms": kernel, "particle_steps_per_s": steps_taken / (kernel / 1e3),
                        "speedup_vs_f32_kernel": f32_kernel_ms / kernel,
                        "fp64_error": fp64_error(a, ctx, field, grid, parts, horizons=(50, 250))}
        field.close()
    return out


def true_rk4(a, ctx, field, grid, parts, p0, r0, pos, rem, term, stream, steps=3):
    """The same workload with runge_kutta_4_true: four field samples per step
    (the reference's runge_kutta_4 takes one, its system ignoring the state),
    so four times the gathers; throughput and error against the FP64 oracle's
    four-sample RK4."""
    import ctypes as C
    from dpa_b200 import _native as N
    lib = ctx._lib
    opts = N.AdvectOptions(N.INTEGRATORS["runge_kutta_4_true"], float(np.float32(a.step_size)),
                           0, 0, 0, 1)
    times = []
    for i in range(steps + 1):
        pos.copy_(p0)
        rem.copy_(r0)
        ctx.check(lib.dpa_advect_device(ctx.handle, field.handle, C.byref(opts), a.seeds,
                                        C.c_void_p(pos.data_ptr()), C.c_void_p(rem.data_ptr()),
                                        C.c_void_p(term.data_ptr()),
                                        C.c_void_p(stream.cuda_stream)))
        o, k = C.c_float(), C.c_float()
        ctx.check(lib.dpa_context_last_timing(ctx.handle, C.byref(o), C.byref(k)))
        if i:
            times.append(k.value)
    taken = float((a.iterations - rem.cpu().numpy().astype(np.int64)).sum())
    kernel = statistics.mean(times)
    return {"field_samples_per_step": 4, "kernel_ms": kernel,
            "particle_steps_per_s": taken / (kernel / 1e3),
            "algorithmic_bytes_per_step": 4 * BYTES_PER_STEP[a.storage],
            "fp64_error": fp64_error(a, ctx, field, grid, parts, horizons=(50, 250),
                                     integrator="runge_kutta_4_true")}


def _graph_replays(ctx, field, opts, p0, r0, pos, rem, term, stream, steps):
    """Times `steps` replays of the captured order + advection graph, each
    after a device reset of the particle state; returns mean ms per replay."""
    import ctypes as C
    import torch
    lib = ctx._lib
    graph = C.c_void_p()
    n = p0.shape[0]
    ctx.check(lib.dpa_graph_create_advect(ctx.handle, field.handle, C.byref(opts), n,
                                          C.c_void_p(pos.data_ptr()), C.c_void_p(rem.data_ptr()),
                                          C.c_void_p(term.data_ptr()), C.byref(graph)))
    times = []
    try:
        for i in range(steps + 2):
            start = torch.cuda.Event(enable_timing=True)
            end = torch.cuda.Event(enable_timing=True)
            start.record(stream)
            pos.copy_(p0)
            rem.copy_(r0)
            ctx.check(lib.dpa_graph_launch(ctx.handle, graph, C.c_void_p(stream.cuda_stream)))
            end.record(stream)
            end.synchronize()
            if i >= 2:
                times.append(start.elapsed_time(end))
    finally:
        lib.dpa_graph_destroy(ctx.handle, graph)
    return statistics.mean(times)


def systems_forms(a, ctx, grid, p0, r0, pos, rem, term, stream, plain_ms, steps=10):
    """The batched form on the same workload: field in FP16 (and FP32 for
    comparison), launch parameters autotuned on the same seeds and budgets, the order +
    advection sequence replayed from a CUDA graph. Ratios are against this
    run's plain FP32 step (dpa_advect_device, default parameters)."""
    import ctypes as C
    from dpa_b200 import _native as N
    lib = ctx._lib
    out = {}
    saved = N.Tuning()
    ctx.check(lib.dpa_context_get_tuning(ctx.handle, C.byref(saved)))
    for storage in ("f16", "f32"):
        field = ctx.field(grid, storage)
        opts = N.AdvectOptions(N.INTEGRATORS[a.integrator], float(np.float32(a.step_size)),
                               0, 0, 0, 1, 0)
        best = N.Tuning()
        ctx.check(lib.dpa_autotune_advect(ctx.handle, field.handle, C.byref(opts), a.seeds,
                                          C.c_void_p(p0.data_ptr()), C.c_void_p(r0.data_ptr()),
                                          0, C.byref(best)))
        ms = _graph_replays(ctx, field, opts, p0, r0, pos, rem, term, stream, steps)
        taken = float((a.iterations - rem.cpu().numpy().astype(np.int64)).sum())
        out[f"{storage}_autotuned_graph"] = {
            "ms_per_step": ms, "particle_steps_per_s": taken / (ms / 1e3),
            "speedup_vs_plain_f32": plain_ms / ms,
            "tuning": {"claim": best.claim, "blocks_per_sm": best.blocks_per_sm,
                       "order": best.order}}
        ctx.check(lib.dpa_context_set_tuning(ctx.handle, C.byref(saved)))
        field.close()
    return out


def batched_run(a, ctx, stream, sets=64):
    """Many seed sets in one persistent launch: a curl-noise field of
    batch_n^3 (sigma 8, seed 3), 64 seed sets with log-uniform sizes in
    [1e3, 1e6] (scaled to the grid when batch_n < 512) and iterations uniform
    in [200, 4000], RK4 step 0.25, end positions only (recording 16 M curves
    of up to 4000 vertices would be ~0.8 TB of output)."""
    import ctypes as C
    import torch
    from dpa_b200 import _native as N
    from dpa_b200 import fields, seeds
    lib = ctx._lib
    n = a.batch_n
    grid = fields.curl_noise(n, 8.0, 3, device="cuda")
    torch.cuda.empty_cache()
    rng = np.random.default_rng(3)
    scale = (n / 512.0) ** 3
    sizes = np.exp(rng.uniform(np.log(1e3), np.log(1e6), size=sets)) * scale
    sizes = np.maximum(sizes.astype(np.int64), 1)
    iters = rng.integers(200, 4001, size=sets)
    offset, size = seeds.seed_box(grid)
    box = ([0.0] * 3, [float(n - 1)] * 3)
    total = int(sizes.sum())
    pos_h = seeds.generate_random(offset, size, total, 0, aabb=box, seed=3).position
    rem_h = np.repeat(iters, sizes).astype(np.int64)
    set_offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    out = {"grid": n, "sets": sets, "particles": total,
           "iterations": {"min": int(iters.min()), "max": int(iters.max())}}
    p0 = torch.from_numpy(pos_h).cuda()
    r0 = torch.from_numpy(rem_h).cuda()
    pos = torch.empty_like(p0)
    rem = torch.empty_like(r0)
    term = torch.empty(total, dtype=torch.uint8, device="cuda")
    for storage in ("f32", "f16"):
        field = ctx.field(grid, storage)
        opts = N.AdvectOptions(N.INTEGRATORS[a.integrator], float(np.float32(a.step_size)),
                               0, 0, 0, 1, 0)
        set_steps = np.zeros(sets, np.uint64)
        times = []
        for i in range(3):
            pos.copy_(p0)
            rem.copy_(r0)
            start = torch.cuda.Event(enable_timing=True)
            end = torch.cuda.Event(enable_timing=True)
            start.record(stream)
            ctx.check(lib.dpa_advect_batch_device(
                ctx.handle, field.handle, C.byref(opts), sets,
                set_offsets.ctypes.data_as(N._U64P), C.c_void_p(pos.data_ptr()),
                C.c_void_p(rem.data_ptr()), C.c_void_p(term.data_ptr()),
                set_steps.ctypes.data_as(N._U64P) if i == 0 else None,
                C.c_void_p(stream.cuda_stream)))
            end.record(stream)
            end.synchronize()
            if i > 0:
                times.append(start.elapsed_time(end))
        ms = statistics.mean(times)
        steps_total = float(set_steps.sum())
        out[storage] = {"ms_per_batch": ms, "particle_steps": steps_total,
                        "particle_steps_per_s": steps_total / (ms / 1e3),
                        "field_device_bytes": field.device_bytes}
        if storage == "f32":
            # The plain FP32 path on the same particles: one dpa_advect_device
            # call over all of them, default launch parameters.
            plain = []
            for i in range(3):
                pos.copy_(p0)
                rem.copy_(r0)
                start = torch.cuda.Event(enable_timing=True)
                end = torch.cuda.Event(enable_timing=True)
                start.record(stream)
                ctx.check(lib.dpa_advect_device(ctx.handle, field.handle, C.byref(opts), total,
                                                C.c_void_p(pos.data_ptr()),
                                                C.c_void_p(rem.data_ptr()),
                                                C.c_void_p(term.data_ptr()),
                                                C.c_void_p(stream.cuda_stream)))
                end.record(stream)
                end.synchronize()
                if i > 0:
                    plain.append(start.elapsed_time(end))
            out["plain_f32_ms"] = statistics.mean(plain)
        field.close()
    out["f16_batched_vs_plain_f32"] = out["plain_f32_ms"] / out["f16"]["ms_per_batch"]
    del p0, r0, pos, rem, term
    torch.cuda.empty_cache()
    return out


def serving_run(a, ctx, rate=200.0, storage="f16"):
    """The serving configuration: resident 256^3 and 512^3 curl-noise fields
    (sigma 4 / seed 1 and sigma 8 / seed 3) and the double gyre on
    128 x 64 x 64 with 32 time slices, stored in `storage` (the FP16 served
    form by default); Poisson arrivals (seed 4) at `rate`
    requests/s for serve_seconds. Request mix: 10 % FTLE on a 64^3 lattice of
    the 256^3 field; 30 % pathlines through the gyre (start times uniform in
    [0, 5], step 0.002); 60 % on either curl-noise field. Five in nine of the
    pathline and curl-noise requests record curves (half of all requests).
    Seeds are log-uniform in [1e2, 1e6], except for recording requests, whose
    seeds are log-uniform in [1e2, 2e3] so that the returned curves fit host
    memory and the link; iterations uniform in [100, 5000]. Seeds are windows
    of pre-drawn pools so that submitting keeps pace with the arrivals.
    Latency is submit to result; throughput counts particle-steps over the
    wall time of the run. Results are dropped once their times are read."""
    import threading as th
    from dpa_b200 import fields, seeds
    from dpa_b200.serve import Server
    grid = fields.curl_noise(256, 4.0, 1, device="cuda")
    big = fields.curl_noise(512, 8.0, 3, device="cuda")
    gyre = fields.double_gyre()
    resident = [ctx.field(grid, storage), ctx.field(big, storage), ctx.field(gyre, storage)]
    rng = np.random.default_rng(4)
    pools = []
    for g, hi in ((grid, 255.0), (big, 511.0)):
        offset, size = seeds.seed_box(g)
        pools.append(seeds.generate_random(offset, size, 2_000_000, 0,
                                           aabb=([0.0] * 3, [hi] * 3), seed=4).position)
    gyre_hi = gyre.offset + gyre.spacing * (np.array(gyre.shape) - 1)
    gyre_pool = (gyre.offset + np.random.default_rng(5).random((2_000_000, 3)) *
                 (gyre_hi - gyre.offset) * 0.999).astype(np.float32)
    offset, size = seeds.seed_box(grid)
    lattice = seeds.generate(offset, size, grid.spacing * np.float32(4), 0).position
    plan = []  # (time, field index, seeds, iterations, record, ftle, start time, step)
    t = 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > a.serve_seconds:
            break
        kind = rng.random()
        iters = int(rng.integers(100, 5001))
        if kind < 0.1:
            plan.append((t, 0, lattice, iters, False, True, 0.0, a.step_size))
            continue
        record = rng.random() < 5.0 / 9.0
        hi = 2e3 if record else 1e6
        count = int(np.exp(rng.uniform(np.log(1e2), np.log(hi))))
        if kind < 0.4:
            start = int(rng.integers(0, len(gyre_pool) - count))
            plan.append((t, 2, gyre_pool[start:start + count], iters, record, False,
                         float(rng.uniform(0.0, 5.0)), 0.002))
            continue
        which = int(rng.integers(0, 2))
        start = int(rng.integers(0, len(pools[which]) - count))
        plan.append((t, which, pools[which][start:start + count], iters, record, False, 0.0,
                     a.step_size))
    results = []
    with Server(ctx, particle_capacity=12_000_000, vertex_capacity=600_000_000,
                steps_per_tick=64, max_requests=1024) as server:
        fids = [server.add_field(f) for f in resident]
        done = th.Event()

        def collect():
            while len(results) < len(plan):
                r = server.poll(wait_ms=50)
                if r is not None:
                    # Keep the times, drop the arrays (a minute of recording
                    # requests returns tens of GB of curves).
                    results.append(types.SimpleNamespace(
                        id=r.id, latency=r.latency, queued=r.queued, admitted=r.admitted,
                        finished=r.finished, particle_steps=r.particle_steps))
                elif done.is_set() and server.stats()["completed"] >= len(plan) and \
                        len(results) >= len(plan):
                    break
        poller = th.Thread(target=collect, daemon=True)
        poller.start()
        t0 = time.perf_counter()
        for when, which, pos, iters, record, ftle, start_time, step in plan:
            delay = when - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            server.submit(fids[which], pos, iters, a.integrator, step, record=record, ftle=ftle,
                          seed_stride=(4.0, 4.0, 4.0), start_time=start_time)
        done.set()
        poller.join(timeout=600)
        wall = time.perf_counter() - t0
        stats = server.stats()
    for f in resident:
        f.close()
    lat = np.array([r.latency for r in results]) * 1e3
    steps = float(sum(r.particle_steps for r in results))
    kinds = {"ftle": sum(1 for p in plan if p[5]), "recording": sum(1 for p in plan if p[4]),
             "pathlines": sum(1 for p in plan if p[1] == 2),
             "on_512": sum(1 for p in plan if p[1] == 1)}

    def pct(values):
        v = np.asarray(values, np.float64) * 1e3
        return {"p50": float(np.percentile(v, 50)), "p99": float(np.percentile(v, 99))} \
            if len(v) else None

    # Kind of each result by its id (ids are handed out in submission order).
    kind_of = {}
    for i, (_, which, _, _, record, ftle, _, _) in enumerate(plan):
        kind_of[i + 1] = ("ftle" if ftle else "pathlines" if which == 2 else
                          "recording" if record else "end_positions")
    by_kind = {}
    for k in ("end_positions", "recording", "pathlines", "ftle"):
        rs = [r for r in results if kind_of.get(r.id) == k]
        by_kind[k] = {"latency_ms": pct([r.latency for r in rs]),
                      "queue_wait_ms": pct([r.admitted - r.queued for r in rs]),
                      "service_ms": pct([r.finished - r.admitted for r in rs])}
    return {"requests": len(plan), "completed": len(results), "rate_per_s": rate,
            "field_storage": storage,
            "seconds_of_arrivals": a.serve_seconds, "wall_seconds": wall,
            "latency_ms": {"p50": float(np.percentile(lat, 50)),
                           "p99": float(np.percentile(lat, 99)), "max": float(lat.max())},
            "queue_wait_ms": pct([r.admitted - r.queued for r in results]),
            "by_kind": by_kind,
            "particle_steps_per_s": steps / wall, "ticks": int(stats["ticks"]),
            "launches": int(stats["launches"]), "busy_seconds": float(stats["busy_seconds"]),
            "tick_device_seconds": float(stats["tick_device_seconds"]),
            "mix": kinds}


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    device = "cuda" if _cuda_available() else None
    grid, parts = make_inputs(a, 0, device)
    per_step = max(2.0, min(8.0, 150.0 / max(a.steps + a.warmup, 1)))
    for _ in range(a.warmup):
        cpu_baseline(a, grid, parts, per_step / 4)
    values, samples = [], []
    for _ in range(a.steps):
        b = cpu_baseline(a, grid, parts, per_step)
        values.append(b["value"])
        samples.append(b["sample"])
    value = statistics.mean(values)
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(a, 1),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                         "sample": samples[-1]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference cannot be built here (Boost, Eigen, TBB, HDF5, MPI absent); this "
                "arm times oracle/oracle.cpp, its reference-faithful C++ restatement",
    }
    print(json.dumps(out), flush=True)
    return 0


def _cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def run_gpu(a):
    import ctypes as C
    import torch
    import torch.distributed as dist
    import dpa_b200
    from dpa_b200 import _native as N

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    grid, parts = make_inputs(a, rank, "cuda")
    ctx = dpa_b200.Context(local)
    lib = ctx._lib
    field = ctx.field(grid, a.storage)
    n = a.seeds
    pristine_pos = torch.from_numpy(parts.position).cuda()
    pristine_rem = torch.full((n,), a.iterations, dtype=torch.int64, device="cuda")
    pos = torch.empty_like(pristine_pos)
    rem = torch.empty_like(pristine_rem)
    term = torch.empty(n, dtype=torch.uint8, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    opts = N.AdvectOptions(N.INTEGRATORS[a.integrator], float(np.float32(a.step_size)), 0, 0, 0, 1)
    # A dedicated stream: torch's default stream is the legacy NULL stream,
    # which the library reads as "use the context's own stream".
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.check(lib.dpa_context_set_profiling(ctx.handle, 1))

    def one_step():
        pos.copy_(pristine_pos)
        rem.copy_(pristine_rem)
        ctx.check(lib.dpa_advect_device(ctx.handle, field.handle, C.byref(opts), n,
                                        C.c_void_p(pos.data_ptr()), C.c_void_p(rem.data_ptr()),
                                        C.c_void_p(term.data_ptr()), C.c_void_p(stream.cuda_stream)))

    for _ in range(a.warmup):
        flush.fill_(1)
        one_step()
    torch.cuda.synchronize()

    launches0 = C.c_uint64()
    ctx.check(lib.dpa_context_launch_count(ctx.handle, C.byref(launches0)))
    clocks = ClockSampler(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    total_ms, kernel_ms, order_ms = 0.0, [], []
    for _ in range(a.steps):
        flush.fill_(2)
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        one_step()
        end.record(stream)
        end.synchronize()
        total_ms += start.elapsed_time(end)
        o, k = C.c_float(), C.c_float()
        ctx.check(lib.dpa_context_last_timing(ctx.handle, C.byref(o), C.byref(k)))
        order_ms.append(o.value)
        kernel_ms.append(k.value)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clock_info = clocks.stop()
    launches1 = C.c_uint64()
    ctx.check(lib.dpa_context_launch_count(ctx.handle, C.byref(launches1)))
    gpu_launches = int(launches1.value - launches0.value)

    rem_out = rem.cpu().numpy().astype(np.int64)
    steps_taken = float(np.sum(a.iterations - rem_out))
    ms_per_step = total_ms / a.steps
    ms_max, steps_total = combine_over_ranks(ms_per_step, steps_taken, "cuda")
    value = steps_total / (ms_max / 1e3)
    gpu_final = pos.cpu().numpy()

    # End to end through the host C ABI with pinned host buffers.
    host_pos = torch.empty((n, 3), dtype=torch.float32, pin_memory=True).numpy()
    host_rem = torch.empty(n, dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
    host_term = torch.empty(n, dtype=torch.uint8, pin_memory=True).numpy()
    e2e_steps = max(1, min(a.steps, 3))
    e2e_opts = N.AdvectOptions(N.INTEGRATORS[a.integrator], float(np.float32(a.step_size)), 0, 0, 0, 1)

    def e2e_once():
        host_pos[:] = parts.position
        host_rem[:] = a.iterations
        t0 = time.perf_counter()
        ctx.check(lib.dpa_advect_round(ctx.handle, field.handle, C.byref(e2e_opts), n,
                                       host_pos.ctypes.data_as(C.c_void_p),
                                       host_rem.ctypes.data_as(C.c_void_p),
                                       host_term.ctypes.data_as(C.c_void_p), N.CURVE_SINK(), None))
        return time.perf_counter() - t0

    e2e_once()
    e2e_times = [e2e_once() for _ in range(e2e_steps)]
    e2e_steps_taken = float(np.sum(a.iterations - host_rem.astype(np.int64)))
    e2e_max, e2e_total = combine_over_ranks(statistics.mean(e2e_times), e2e_steps_taken, "cuda")
    e2e_value = e2e_total / e2e_max

    peak, peak_src = measured_peak_hbm()
    kernel_s = statistics.mean(kernel_ms) / 1e3
    algorithmic = BYTES_PER_STEP[a.storage] * steps_taken + STATE_BYTES * n
    achieved = algorithmic / kernel_s / 1e9
    traffic = None
    tf = ROOT / "profiles" / "advect_traffic.json"
    # The captured traffic is that of the default workload's launch (1,048,576
    # seeds x 2000 iterations of step 0.25); other workloads have none.
    if tf.exists() and a.seeds == 1 << 20 and a.iterations == 2000 and a.step_size == 0.25:
        try:
            traffic = json.loads(tf.read_text()).get(f"{a.storage}_{a.integrator}_n{a.n}")
        except Exception:
            traffic = None

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(a, world),
        "particle_steps_per_step": steps_total,
        "kernel_ms": statistics.mean(kernel_ms), "order_ms": statistics.mean(order_ms),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "dram_achieved": traffic / kernel_s / 1e9 if traffic else None,
                     "peak_source": peak_src,
                     "algorithmic_bytes": f"{BYTES_PER_STEP[a.storage]} B per particle-step "
                                          f"(8 corners x 3 x {BYTES_PER_STEP[a.storage] // 24} B)"
                                          f" + {STATE_BYTES} B particle state per particle",
                     "kernel": "advect_kernel (CUDA events around its launch, on its stream)"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": n * (12 + 8),
                "d2h_bytes_per_step": n * (12 + 8 + 1),
                "call": "dpa_advect_round with pinned host buffers (wall clock around the "
                        "synchronous call)"},
        "gpu_launches": gpu_launches,
        "clocks": clock_info,
    }
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(a, grid, parts, a.cpu_seconds)
        out["fp64_error"] = fp64_error(a, ctx, field, grid, parts)
        out["precision_forms"] = precision_forms(a, ctx, grid, parts, pristine_pos, pristine_rem,
                                                 pos, rem, term, stream, statistics.mean(kernel_ms))
        out["true_rk4"] = true_rk4(a, ctx, field, grid, parts, pristine_pos, pristine_rem, pos,
                                   rem, term, stream)
        if not a.no_systems:
            out["systems_forms"] = systems_forms(a, ctx, grid, pristine_pos, pristine_rem, pos, rem,
                                                 term, stream, ms_max)
            out["batched"] = batched_run(a, ctx, stream)
            out["serving"] = serving_run(a, ctx)
    if rank == 0:
        print(json.dumps(out), flush=True)
    field.close()
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


SECONDARY = {
    # workload: field, seeds, iterations, step, what a step does
    "ftle": "ABC flow + 5 % smoothed perturbation (sigma 3, seed 2) on 256^3 over [0, 2 pi]^3, "
            "a 128^3 seed lattice (seed_generation_stride 2), runge_kutta_4 (one field sample "
            "per step), step 0.02, 250 iterations, then the FTLE of the flow map",
    "recording": "ABC flow on 64^3 over [0, 2 pi]^3, 4096 uniform seeds (seed 0) in the domain, "
                 "runge_kutta_4 (one field sample per step), step 0.01, 1000 iterations, curve "
                 "recording with uint32 indices and angular-velocity colors",
}


def secondary_inputs(a, device):
    import math
    from dpa_b200 import fields, seeds
    if a.workload == "ftle":
        grid = fields.abc_perturbed(256, 0.05, 3.0, 2, device=device)
        offset, size = seeds.seed_box(grid)
        parts = seeds.generate(offset, size, (grid.spacing * np.float32(2)).astype(np.float32), 250)
        return grid, parts.position, 250, 0.02
    grid = fields.abc(64)
    offset, size = seeds.seed_box(grid)
    parts = seeds.generate_random(offset, size, 4096, 1000, aabb=([0, 0, 0], [2 * math.pi] * 3),
                                  seed=0)
    return grid, parts.position, 1000, 0.01


def recording_at_scale(ctx, a, n=262144, iterations=2000):
    """Curve recording at scale: the 256^3 curl-noise field, n seeds x
    `iterations` steps of 0.25, through dpa_advect_round with a sink that
    takes each chunk without copying it (the curves -- vertices, colors,
    indices -- still cross to pinned host memory). uint32 and uint64
    indices."""
    import ctypes as C
    from dpa_b200 import _native as N
    from dpa_b200 import fields, seeds
    lib = ctx._lib
    grid = fields.curl_noise(256, 4.0, 1, device="cuda")
    field = ctx.field(grid)
    offset, size = seeds.seed_box(grid)
    pos = seeds.generate_random(offset, size, n, 0, aabb=([0.0] * 3, [255.0] * 3), seed=1).position
    totals = {"vertices": 0, "indices": 0}

    @N.CURVE_SINK
    def sink(user, chunk):
        totals["vertices"] += chunk.contents.vertex_count
        totals["indices"] += chunk.contents.index_count
        return 0

    out = {"workload": f"curl-noise 256^3 F32, {n} seeds x {iterations} steps of 0.25, recording",
           "sink": "takes each chunk in place (no copy)"}
    for index64 in (0, 1):
        opts = N.AdvectOptions(N.INTEGRATORS[a.integrator], 0.25, 1, index64, 1, 1, 0)
        times = []
        for _ in range(3):
            hp, hr = pos.copy(), np.full(n, iterations, np.uint64)
            ht = np.zeros(n, np.uint8)
            totals.update(vertices=0, indices=0)
            t0 = time.perf_counter()
            ctx.check(lib.dpa_advect_round(ctx.handle, field.handle, C.byref(opts), n,
                                           hp.ctypes.data_as(C.c_void_p),
                                           hr.ctypes.data_as(C.c_void_p),
                                           ht.ctypes.data_as(C.c_void_p), sink, None))
            times.append(time.perf_counter() - t0)
        t = min(times)
        steps = float(np.sum(iterations - hr.astype(np.int64)))
        gb = (totals["vertices"] * 16 + totals["indices"] * (8 if index64 else 4)) / 1e9
        out["uint64" if index64 else "uint32"] = {
            "seconds": t, "particle_steps_per_s": steps / t, "vertices": totals["vertices"],
            "indices": totals["indices"], "curve_GB": gb, "curve_GB_per_s": gb / t}
    field.close()
    return out


def ftle_fp64_error(grid, lattice, ftle_by_storage, iterations, step, lo=60, m=16):
    """FTLE error against the FP64 oracle on an m^3 block of interior lattice
    cells starting at lattice index lo (clear of the planes where the
    reference's cell mapping collides): the block and a one-cell halo are
    advected in double (the reference's one-sample RK4), the flow-map
    Jacobian is taken by central differences over the lattice spacing, and
    FTLE = ln sqrt(lambda_max(J^T J)) / |step * iterations|. Returns the
    relative error of each storage's GPU FTLE over the block."""
    from oracle import binding as ob
    ob.build()
    ob.set_threads(os.cpu_count() or 1)
    n = 128
    idx = np.arange(lo - 1, lo + m + 1)
    ii, jj, kk = np.meshgrid(idx, idx, idx, indexing="ij")
    flat = (ii * n + jj) * n + kk
    seeds = lattice[flat.reshape(-1)]
    r = ob.advect64(ob.OracleGrid.of(grid), "runge_kutta_4", step, seeds,
                    np.full(len(seeds), iterations, np.uint64))
    flow = r.positions.reshape(m + 2, m + 2, m + 2, 3)
    h = 2.0 * np.asarray(grid.spacing, np.float64) * 2.0  # central difference over 2 lattice cells
    J = np.stack([(flow[2:, 1:-1, 1:-1] - flow[:-2, 1:-1, 1:-1]) / h[0],
                  (flow[1:-1, 2:, 1:-1] - flow[1:-1, :-2, 1:-1]) / h[1],
                  (flow[1:-1, 1:-1, 2:] - flow[1:-1, 1:-1, :-2]) / h[2]], axis=-1)
    C = np.einsum("...ki,...kj->...ij", J, J)
    lam = np.linalg.eigvalsh(C)[..., -1]
    want = np.log(np.sqrt(lam)) / abs(float(np.float32(step) * np.float32(iterations)))
    # Cells whose whole stencil ran every iteration without leaving the grid:
    # elsewhere the flow map holds exit positions, which a one-step difference
    # in the exit moves by a cell or more.
    done = (r.termination == 0).reshape(m + 2, m + 2, m + 2)
    inside = done[1:-1, 1:-1, 1:-1].copy()
    for d, sl in enumerate([(slice(2, None), slice(1, -1), slice(1, -1)),
                            (slice(None, -2), slice(1, -1), slice(1, -1)),
                            (slice(1, -1), slice(2, None), slice(1, -1)),
                            (slice(1, -1), slice(None, -2), slice(1, -1)),
                            (slice(1, -1), slice(1, -1), slice(2, None)),
                            (slice(1, -1), slice(1, -1), slice(None, -2))]):
        inside &= done[sl]
    out = {"block": f"lattice cells [{lo}, {lo + m})^3 of 128^3, FP64 reference-semantics RK4"}
    for storage, ftle in ftle_by_storage.items():
        got = ftle.reshape(n, n, n)[lo:lo + m, lo:lo + m, lo:lo + m].astype(np.float64)
        ok = np.isfinite(want) & np.isfinite(got) & (np.abs(want) > 1e-6)
        entry = {}
        for name, mask in (("all_cells", ok), ("stencil_inside", ok & inside)):
            if not mask.any():
                entry[name] = {"cells": 0}
                continue
            rel = np.abs(got[mask] - want[mask]) / np.abs(want[mask])
            entry[name] = {"cells": int(mask.sum()), "median_rel": float(np.median(rel)),
                           "p99_rel": float(np.percentile(rel, 99)), "max_rel": float(rel.max())}
        out[storage] = entry
    return out


def run_secondary(a):
    """The FTLE and recording configurations: device-timed steps through the
    device entry points (FTLE) or the host round with its curve (recording),
    in the same JSON layout as the headline workload."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if a.impl == "reference":
        if rank != 0:
            return 0
        grid, pos, iterations, step = secondary_inputs(a, "cuda" if _cuda_available() else None)
        from oracle import binding as ob
        ob.build()
        threads = os.cpu_count() or 1
        ob.set_threads(threads)
        og = ob.OracleGrid.of(grid)
        values = []
        sample = pos
        if a.workload == "ftle":  # a seeded random sample of the lattice, ~5 s of work
            sample = pos[np.sort(np.random.default_rng(11).choice(len(pos), 200_000, False))]
        for i in range(a.warmup + a.steps):
            t0 = time.perf_counter()
            r = ob.advect_round(og, a.integrator, step, sample,
                                np.full(len(sample), iterations, np.uint64),
                                record=a.workload == "recording")
            dt = time.perf_counter() - t0
            if i >= a.warmup:
                values.append(float(np.sum(r.steps)) / dt)
        value = statistics.mean(values)
        desc = (f"{len(sample)} of the {len(pos)} seeds at full {iterations} iterations per step; "
                "oracle/oracle.cpp, OpenMP dynamic schedule standing in for TBB")
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": SECONDARY[a.workload]},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}), flush=True)
        return 0

    import ctypes as C
    import torch
    import dpa_b200
    from dpa_b200 import ParticleAdvector, Particles
    from dpa_b200 import _native as N
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    grid, pos, iterations, step = secondary_inputs(a, "cuda")
    n = pos.shape[0]
    ctx = dpa_b200.Context(local)
    lib = ctx._lib
    field = ctx.field(grid, a.storage)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    clocks = ClockSampler(local)
    out = {"metric": METRIC, "unit": UNIT, "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic",
           "config": {"workload": SECONDARY[a.workload], "storage": a.storage,
                      "l2": "256 MiB buffer written between timed steps (L2 flush)"}}
    launches0 = C.c_uint64()
    ctx.check(lib.dpa_context_launch_count(ctx.handle, C.byref(launches0)))
    if a.workload == "ftle":
        p0 = torch.from_numpy(pos).cuda()
        r0 = torch.full((n,), iterations, dtype=torch.int64, device="cuda")
        p, r = torch.empty_like(p0), torch.empty_like(r0)
        term = torch.empty(n, dtype=torch.uint8, device="cuda")
        stride = (C.c_float * 3)(2.0, 2.0, 2.0)
        shape = (C.c_uint64 * 3)()
        ftle = torch.empty(128 ** 3, dtype=torch.float32, device="cuda")
        opts = N.AdvectOptions(N.INTEGRATORS[a.integrator], float(np.float32(step)), 0, 0, 0, 1)
        ctx.check(lib.dpa_context_set_profiling(ctx.handle, 1))
        kernel_ms, ftle_ms, total = [], [], 0.0

        def one_step():
            p.copy_(p0)
            r.copy_(r0)
            ctx.check(lib.dpa_advect_device(ctx.handle, field.handle, C.byref(opts), n,
                                            C.c_void_p(p.data_ptr()), C.c_void_p(r.data_ptr()),
                                            C.c_void_p(term.data_ptr()),
                                            C.c_void_p(stream.cuda_stream)))
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.check(lib.dpa_ftle_estimate_device(
                ctx.handle, field.handle, stride, iterations, float(np.float32(step)), n,
                C.c_void_p(p0.data_ptr()), C.c_void_p(p.data_ptr()), 0,
                C.c_void_p(ftle.data_ptr()), shape, C.c_void_p(stream.cuda_stream)))
            e1.record(stream)
            return e0, e1

        for _ in range(a.warmup):
            flush.fill_(1)
            one_step()
        torch.cuda.synchronize()
        ctx.check(lib.dpa_context_launch_count(ctx.handle, C.byref(launches0)))
        clocks.start()
        time.sleep(0.3)  # the sampler's first readings
        for _ in range(a.steps):
            flush.fill_(2)
            start = torch.cuda.Event(enable_timing=True)
            end = torch.cuda.Event(enable_timing=True)
            start.record(stream)
            e0, e1 = one_step()
            end.record(stream)
            end.synchronize()
            total += start.elapsed_time(end)
            o, k = C.c_float(), C.c_float()
            ctx.check(lib.dpa_context_last_timing(ctx.handle, C.byref(o), C.byref(k)))
            kernel_ms.append(k.value)
            ftle_ms.append(e0.elapsed_time(e1))
        out["clocks"] = clocks.stop()
        steps_taken = float(np.sum(iterations - r.cpu().numpy()))
        ms = total / a.steps
        kern = statistics.mean(kernel_ms)
        # End to end: the host entry points (dpa_advect_round, dpa_ftle_estimate)
        # with pinned host buffers.
        hp = torch.empty((n, 3), dtype=torch.float32, pin_memory=True).numpy()
        hr = torch.empty(n, dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
        ht = torch.empty(n, dtype=torch.uint8, pin_memory=True).numpy()
        hf = torch.empty(128 ** 3, dtype=torch.float32, pin_memory=True).numpy()
        hsh = (C.c_uint64 * 3)()

        def e2e_once():
            hp[:] = pos
            hr[:] = iterations
            t0 = time.perf_counter()
            ctx.check(lib.dpa_advect_round(ctx.handle, field.handle, C.byref(opts), n,
                                           hp.ctypes.data_as(C.c_void_p),
                                           hr.ctypes.data_as(C.c_void_p),
                                           ht.ctypes.data_as(C.c_void_p), N.CURVE_SINK(), None))
            ctx.check(lib.dpa_ftle_estimate(ctx.handle, field.handle, stride, iterations,
                                            float(np.float32(step)), n,
                                            pos.ctypes.data_as(C.c_void_p),
                                            hp.ctypes.data_as(C.c_void_p), 0,
                                            hf.ctypes.data_as(C.c_void_p), hsh))
            return time.perf_counter() - t0

        e2e_once()
        e2e = statistics.mean([e2e_once() for _ in range(3)])
        # FTLE of the other storage on the same lattice, and both against
        # the FP64 oracle on an interior block.
        ftles = {a.storage: ftle.cpu().numpy()}
        other = "f16" if a.storage == "f32" else "f32"
        f2 = ctx.field(grid, other)
        p.copy_(p0)
        r.copy_(r0)
        ctx.check(lib.dpa_advect_device(ctx.handle, f2.handle, C.byref(opts), n,
                                        C.c_void_p(p.data_ptr()), C.c_void_p(r.data_ptr()),
                                        C.c_void_p(term.data_ptr()),
                                        C.c_void_p(stream.cuda_stream)))
        ctx.check(lib.dpa_ftle_estimate_device(
            ctx.handle, f2.handle, stride, iterations, float(np.float32(step)), n,
            C.c_void_p(p0.data_ptr()), C.c_void_p(p.data_ptr()), 0,
            C.c_void_p(ftle.data_ptr()), shape, C.c_void_p(stream.cuda_stream)))
        ftles[other] = ftle.cpu().numpy()
        f2.close()
        out["ftle_fp64_error"] = ftle_fp64_error(grid, pos, ftles, iterations, step)
        out.update({
            "value": steps_taken / (ms / 1e3), "ms_per_step": ms,
            "particle_steps_per_step": steps_taken, "kernel_ms": kern,
            "ftle_ms": statistics.mean(ftle_ms),
            "e2e": {"value": steps_taken / e2e, "unit": UNIT,
                    "h2d_bytes_per_step": n * (12 + 8) + n * 24,
                    "d2h_bytes_per_step": n * (12 + 8 + 1) + 128 ** 3 * 4,
                    "call": "dpa_advect_round + dpa_ftle_estimate with pinned host buffers"},
        })
        algorithmic = BYTES_PER_STEP[a.storage] * steps_taken + STATE_BYTES * n
    else:
        adv = ParticleAdvector(ctx, n, "none", a.integrator, step, False, True)
        parts = Particles.create(pos, iterations)
        for _ in range(a.warmup):
            adv.advect(field, parts)
        torch.cuda.synchronize()
        ctx.check(lib.dpa_context_launch_count(ctx.handle, C.byref(launches0)))
        clocks.start()
        time.sleep(0.3)  # the sampler's first readings
        times = []
        for _ in range(a.steps):
            flush.fill_(2)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = adv.advect(field, parts)
            times.append(time.perf_counter() - t0)
        out["clocks"] = clocks.stop()
        curve = res.integral_curves[0]
        steps_taken = float(np.sum(iterations - res.inactive_particles.remaining_iterations
                                   .astype(np.int64)))
        ms = statistics.mean(times) * 1e3
        vertices = int(curve.vertices.shape[0])
        out.update({
            "value": steps_taken / (ms / 1e3), "ms_per_step": ms,
            "particle_steps_per_step": steps_taken,
            "curve": {"vertices": vertices, "indices": int(curve.indices.size),
                      "index_dtype": str(curve.indices.dtype)},
            "e2e": {"value": steps_taken / (ms / 1e3), "unit": UNIT,
                    "h2d_bytes_per_step": n * (12 + 8),
                    "d2h_bytes_per_step": n * (12 + 8 + 1) + vertices * 16 +
                                          int(curve.indices.nbytes),
                    "call": "ParticleAdvector.advect -> dpa_advect_round with recording "
                            "(host buffers, curve chunks through the sink); the timed step "
                            "is this end-to-end call"},
        })
        algorithmic = None
        # Positions against the FP64 oracle integrator, every seed, at
        # horizons most seeds still live to (half have left the domain by
        # step 100, nearly all by step 500).
        config = types.SimpleNamespace(integrator=a.integrator, step_size=step,
                                       iterations=iterations)
        out["fp64_error"] = fp64_error(config, ctx, field, grid, parts, sample=n,
                                       horizons=(50, 100, 250))
        out["at_scale"] = recording_at_scale(ctx, a)
    launches1 = C.c_uint64()
    ctx.check(lib.dpa_context_launch_count(ctx.handle, C.byref(launches1)))
    out["gpu_launches"] = int(launches1.value - launches0.value)
    peak, peak_src = measured_peak_hbm()
    if algorithmic is not None:
        kernel_s = out["kernel_ms"] / 1e3
        achieved = algorithmic / kernel_s / 1e9
        out["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                           "frac": achieved / peak, "traffic": None, "peak_source": peak_src,
                           "algorithmic_bytes": f"{BYTES_PER_STEP[a.storage]} B per "
                                                f"particle-step + {STATE_BYTES} B per particle",
                           "kernel": "advect_kernel (CUDA events around its launch)"}
    print(json.dumps(out), flush=True)
    field.close()
    ctx.close()
    return 0


def main():
    a = parse_args()
    if a.workload != "throughput":
        return run_secondary(a)
    if a.impl == "reference":
        return run_reference(a)
    return run_gpu(a)


if __name__ == "__main__":
    sys.exit(main())
