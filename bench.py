#!/usr/bin/env python
"""Throughput of the advection hot path on the B200, one JSON line.

Headline workload (the throughput configuration): a 256^3 FP32 curl-noise
field (sigma 4 cells, field seed 1, spacing 1, unit RMS speed), 1,048,576
seeds uniform in the valid domain [0, 255)^3 (seed 1; rank r uses seed
1 + r), runge_kutta_4 with the reference's semantics, step 0.25, 2000
iterations, end positions only. One bench step advects every seed through
all its iterations: particle state reset on the device, processing order,
advection.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

`value` is whole-job particle-steps/s (steps actually taken, summed over
ranks, divided by the max over ranks of the device-timed step). `e2e` is the
same metric through the host C ABI call (dpa_advect_round) with pinned host
buffers, copies included. The CPU baseline is the oracle's reference-faithful
restatement on a bounded seed sample on the host cores.

The same line carries the other configurations, each with its own device
rate, end-to-end rate, CPU baseline timed in this run and error against the
FP64 oracle: `recording` (64^3 ABC, 4096 seeds x 1000 steps, curves with
uint32 indices), `ftle` (256^3 ABC + noise, 128^3 lattice x 250 steps, FTLE),
`batched` (512^3 curl noise, 64 seed sets, 16 M particles, recording with
uint64 indices, graph-captured autotuned launches) and `serving` (resident
fields, Poisson arrivals, p50/p99 latency over three seeded runs).
`--workload NAME` prints one of them alone.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
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
BYTES_PER_STEP = {"f32": 96, "f16": 48, "bf16": 48, "f32_edges": 96}  # 8 corners x 3 components
STATE_BYTES = 12 + 8 + 12 + 8 + 1  # positions + remaining in, out + termination
TRAFFIC_FILE = ROOT / "profiles" / "advect_traffic.json"


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=30)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="dpa_b200", choices=["dpa_b200", "reference"])
    p.add_argument("--workload", default="throughput",
                   choices=["throughput", "recording", "ftle", "batched", "serving"],
                   help="throughput: the headline line with every configuration; the others "
                        "print one configuration alone")
    p.add_argument("--storage", default="f32", choices=["f32", "f16", "bf16", "f32_edges"])
    p.add_argument("--integrator", default="runge_kutta_4")
    p.add_argument("--grid", dest="n", type=int, default=256,
                   help="grid points per axis of the throughput workload")
    p.add_argument("--seeds", type=int, default=1 << 20)
    p.add_argument("--iterations", type=int, default=2000)
    p.add_argument("--step-size", type=float, default=0.25)
    p.add_argument("--cpu-seconds", type=float, default=10.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-systems", action="store_true",
                   help="skip the other configurations (recording, FTLE, batched, serving)")
    p.add_argument("--serve-seconds", type=float, default=20.0,
                   help="seconds of Poisson arrivals in each serving run")
    p.add_argument("--serve-runs", type=int, default=3, help="seeded serving runs (seeds 4, 5, ...)")
    p.add_argument("--batch-n", type=int, default=512)
    p.add_argument("--batch-particles", type=int, default=1 << 24)
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
            self.lines.append((time.perf_counter(), line.strip()))

    def stop(self, window=None) -> dict:
        """Median SM clock and the throttle reasons seen; with window = (t0,
        t1) (perf_counter times of the timed region), only the samples taken
        in it (or, when it is shorter than the sampling period, the three
        nearest)."""
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        lines = self.lines
        if window and lines:
            t0, t1 = window
            inside = [x for x in lines if t0 - 0.05 <= x[0] <= t1 + 0.05]
            if len(inside) < 3:
                mid = 0.5 * (t0 + t1)
                inside = sorted(lines, key=lambda x: abs(x[0] - mid))[:3]
            lines = inside
        sms, maxes, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for _, line in lines:
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


def _oracle():
    from oracle import binding as ob
    ob.build()
    ob.set_threads(os.cpu_count() or 1)
    return ob


def cpu_rate(grid, integrator, step, positions, remaining, target_seconds, record=False,
             max_count=None, describe=""):
    """The oracle's reference-faithful restatement (oracle/oracle.cpp, OpenMP
    dynamic schedule standing in for TBB) on all host threads, on the first
    seeds of `positions` sized for about `target_seconds` of work (or all of
    them, up to max_count)."""
    ob = _oracle()
    threads = os.cpu_count() or 1
    og = ob.OracleGrid.of(grid)
    total = positions.shape[0] if max_count is None else min(max_count, positions.shape[0])
    calib = min(total, max(threads * 8, 64))
    t0 = time.perf_counter()
    r = ob.advect_round(og, integrator, step, positions[:calib], remaining[:calib], record=record)
    dt = time.perf_counter() - t0
    rate = float(np.sum(r.steps)) / max(dt, 1e-9)
    per = max(float(np.mean(r.steps)), 1.0)
    count = int(min(total, max(calib, rate * target_seconds / per)))
    t0 = time.perf_counter()
    r = ob.advect_round(og, integrator, step, positions[:count], remaining[:count], record=record)
    dt = time.perf_counter() - t0
    taken = float(np.sum(r.steps))
    return {"value": taken / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"first {count} of {positions.shape[0]} seeds at full iterations "
                      f"({int(taken)} particle-steps in {dt:.2f} s{', recording' if record else ''}"
                      f"{describe}; oracle/oracle.cpp, OpenMP dynamic schedule standing in for "
                      "TBB)"}


def cpu_baseline(a, grid, parts, target_seconds):
    return cpu_rate(grid, a.integrator, a.step_size, parts.position,
                    np.full(parts.position.shape[0], a.iterations, np.uint64), target_seconds)


def position_error(gpu, ref, spacing):
    ok = (ref.termination == 0) & (gpu.termination == 0)
    err = np.linalg.norm(gpu.position[ok].astype(np.float64) - ref.positions[ok], axis=1)
    err = err / float(spacing)
    return {"completed": int(ok.sum()),
            "median_cells": float(np.median(err)) if ok.any() else None,
            "p99_cells": float(np.percentile(err, 99)) if ok.any() else None,
            "max_cells": float(np.max(err)) if ok.any() else None,
            "within_1e-3_cells": float(np.mean(err <= 1e-3)) if ok.any() else None}


def fp64_error(ctx, field, grid, positions, integrator, step, horizons, sample=512):
    """Position error of the GPU path against the FP64 oracle integrator (the
    same scheme in double), in cells, over the first `sample` seeds that
    complete in both, at several horizons (chaotic fields separate FP32 and
    FP64 trajectories exponentially, so only short horizons measure the
    integrator and the field storage)."""
    from dpa_b200 import ParticleAdvector, Particles
    ob = _oracle()
    og = ob.OracleGrid.of(grid)
    sample = min(sample, positions.shape[0])
    out = {"sample": sample}
    adv = ParticleAdvector(ctx, sample, "none", integrator, step, False, False)
    for h in horizons:
        gpu = adv.advect(field, Particles.create(positions[:sample], h)).inactive_particles
        ref = ob.advect64(og, integrator, step, positions[:sample], np.full(sample, h, np.uint64))
        out[f"steps_{h}"] = position_error(gpu, ref, grid.spacing[0])
    return out


def within_horizon(err, bar=0.99):
    """The longest horizon of `err` at which at least `bar` of the particles
    are within 1e-3 cells of the FP64 oracle (None if none is)."""
    best = None
    for k, v in err.items():
        if k.startswith("steps_") and v.get("within_1e-3_cells") is not None:
            if v["within_1e-3_cells"] >= bar:
                h = int(k[len("steps_"):])
                best = h if best is None else max(best, h)
    return best


KERNEL_SOURCES = ["advect_kernel.cuh", "sample.cuh", "common.cuh", "kernels.cuh", "advect.cu",
                  "advect_f32.cu", "advect_f32e.cu", "advect_f16.cu", "advect_bf16.cu"]


def _code_lines(text):
    """The lines of a source with `//` comments, trailing blanks and empty
    lines removed (the kernel sources hold no `//` inside string literals)."""
    out = []
    for line in text.splitlines():
        code = line.split("//", 1)[0].rstrip()
        if code:
            out.append(code)
    return "\n".join(out)


def kernel_sources_digest():
    """SHA-256 of the code of the sources that make up the advection kernels
    (the figures of a capture depend on these alone; comments do not count)."""
    import hashlib
    h = hashlib.sha256()
    for name in KERNEL_SOURCES:
        h.update(name.encode())
        h.update(_code_lines((ROOT / "dpa_b200" / "csrc" / name).read_text()).encode())
    return h.hexdigest()


def traffic_profile(key):
    """Per-particle-step figures of one workload's advection kernel from the
    committed ncu capture (profiles/advect_traffic.json): DRAM bytes, L1TEX
    bytes and issue activity, with the digest of the kernel sources they were
    captured from and whether the sources here are the same."""
    try:
        d = json.loads(TRAFFIC_FILE.read_text())
    except Exception:
        return None
    entry = d.get("workloads", {}).get(key)
    if not entry:
        return None
    entry = dict(entry)
    try:
        entry["captured_with_current_sources"] = \
            kernel_sources_digest() == d.get("kernel_sources_digest")
    except Exception:
        entry["captured_with_current_sources"] = None
    return entry


def gather_peaks(ctx):
    """Load bandwidth of the gather pattern measured on this device
    (dpa_measure_gather_bandwidth): the L1 data path with coalesced lanes (its
    ceiling), L1-resident random cells and L2-resident random cells."""
    lib = ctx._lib
    out = {}
    for name, nbytes, pattern in (("l1_coalesced", 64 << 10, 0), ("l1_random", 64 << 10, 1),
                                  ("l2_random", 64 << 20, 1)):
        g = C.c_double()
        ctx.check(lib.dpa_measure_gather_bandwidth(ctx.handle, nbytes, pattern, C.byref(g)))
        out[name] = g.value
    return out


def roofline(kernel_s, steps, particles, storage, key, peaks, samples_per_step=1):
    """The advection kernel's roofline: DRAM bytes against the measured HBM
    copy bandwidth (the contract's `bound`; the bytes come from the committed
    ncu capture of this workload, per particle-step, scaled by this run's
    steps), and the resource that saturates first (`limiter`: the L1TEX data
    path, from the same capture, with the load bandwidth of the gather
    pattern measured in this run beside it)."""
    peak, peak_src = measured_peak_hbm()
    prof = traffic_profile(key)
    algorithmic = (BYTES_PER_STEP[storage] * samples_per_step * steps + STATE_BYTES * particles)
    out = {"bound": "hbm", "unit": "GB/s", "peak": peak, "peak_source": peak_src,
           "kernel": "advect_kernel (CUDA events around its launch, on its stream)",
           "algorithmic_gbs": algorithmic / kernel_s / 1e9,
           "algorithmic_bytes": f"{BYTES_PER_STEP[storage] * samples_per_step} B per particle-step "
                                f"(8 corners x 3 components per field sample) + {STATE_BYTES} B "
                                "per particle; the per-lane cell cache, L1 and L2 serve most of "
                                "it, so it is not DRAM traffic"}
    if peaks:
        out["algorithmic_frac_of_l1_peak"] = out["algorithmic_gbs"] / peaks["l1_coalesced"]
    if not prof:
        out.update({"achieved": None, "traffic": None, "frac": None,
                    "traffic_source": "no capture of this workload"})
        return out
    traffic = prof["dram_bytes_per_step"] * steps
    out.update({"achieved": traffic / kernel_s / 1e9, "traffic": traffic,
                "frac": traffic / kernel_s / 1e9 / peak,
                "traffic_source": f"{prof['capture']}: {prof['dram_bytes_per_step']:.2f} DRAM B "
                                  "per particle-step, scaled by this run's steps",
                "captured_with_current_sources": prof["captured_with_current_sources"]})
    if "l1tex_throughput_pct" in prof:
        lim = {"resource": "L1TEX data path (the corner gathers' requests and sectors)",
               "frac": prof["l1tex_throughput_pct"] / 100.0,
               "frac_source": "ncu l1tex__throughput.avg.pct_of_peak_sustained_active",
               "l1_sector_gbs": prof["l1_sector_bytes_per_step"] * steps / kernel_s / 1e9,
               "issue_active_pct": prof["issue_active_pct"],
               "warps_active_pct": prof["warps_active_pct"],
               "long_scoreboard_stalls_per_issue": prof["long_scoreboard_per_issue"],
               "warp_instructions_per_step": prof["warp_instructions_per_step"]}
        if peaks:
            lim["l1_gather_peaks_gbs"] = peaks
        out["limiter"] = lim
    return out


def _graph_replays(ctx, field, opts, p0, r0, pos, rem, term, stream, steps):
    """Times `steps` replays of the captured order + advection graph, each
    after a device reset of the particle state; returns mean ms per replay."""
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
            pos.copy_(p0)
            rem.copy_(r0)
            start.record(stream)
            ctx.check(lib.dpa_graph_launch(ctx.handle, graph, C.c_void_p(stream.cuda_stream)))
            end.record(stream)
            end.synchronize()
            if i >= 2:
                times.append(start.elapsed_time(end))
    finally:
        lib.dpa_graph_destroy(ctx.handle, graph)
    return statistics.mean(times)


def _tuning_dict(t):
    return {"claim": t.claim, "blocks_per_sm": t.blocks_per_sm, "order": t.order,
            "block_size": t.block_size, "particles_per_thread": t.particles_per_thread}


def autotune(ctx, field, opts, p0, r0, count, sample_steps=0):
    from dpa_b200 import _native as N
    best = N.Tuning()
    ctx.check(ctx._lib.dpa_autotune_advect(ctx.handle, field.handle, C.byref(opts), count,
                                           C.c_void_p(p0.data_ptr()), C.c_void_p(r0.data_ptr()),
                                           sample_steps, C.byref(best)))
    return best


def device_steps(ctx, field, opts, p0, r0, stream, reps):
    """Kernel time (library events) of `reps` dpa_advect_device calls over
    p0/r0 (state reset before each), L2 flushed between them."""
    import torch
    lib = ctx._lib
    n = p0.shape[0]
    pos, rem = torch.empty_like(p0), torch.empty_like(r0)
    term = torch.empty(n, dtype=torch.uint8, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    ks = []
    for i in range(reps + 1):
        flush.fill_(i & 1)
        pos.copy_(p0)
        rem.copy_(r0)
        ctx.check(lib.dpa_advect_device(ctx.handle, field.handle, C.byref(opts), n,
                                        C.c_void_p(pos.data_ptr()), C.c_void_p(rem.data_ptr()),
                                        C.c_void_p(term.data_ptr()),
                                        C.c_void_p(stream.cuda_stream)))
        o, k = C.c_float(), C.c_float()
        ctx.check(lib.dpa_context_last_timing(ctx.handle, C.byref(o), C.byref(k)))
        if i:
            ks.append(k.value)
    return statistics.mean(ks), pos, rem, term


def precision_forms(a, ctx, grid, parts, p0, r0, stream, f32_kernel_ms):
    """The same workload with the field stored in FP16 and BF16 (FP32
    interpolation and accumulation): kernel time, speed-up over this run's
    FP32 kernel, and position error against the FP64 oracle at 10 to 250
    steps, with the longest horizon at which 99 % of the particles stay within
    1e-3 cells (and the same for the FP32 field)."""
    from dpa_b200 import _native as N
    out = {}
    horizons = (10, 25, 50, 100, 250)
    for storage in ("f32", "f16", "bf16"):
        field = ctx.field(grid, storage)
        entry = {}
        if storage != a.storage:
            opts = N.AdvectOptions(N.INTEGRATORS[a.integrator], float(np.float32(a.step_size)),
                                   0, 0, 0, 1, 0)
            kernel, _, rem, _ = device_steps(ctx, field, opts, p0, r0, stream, 5)
            taken = float((a.iterations - rem.cpu().numpy().astype(np.int64)).sum())
            entry.update({"kernel_ms": kernel, "particle_steps_per_s": taken / (kernel / 1e3),
                          "speedup_vs_f32_kernel": f32_kernel_ms / kernel})
        err = fp64_error(ctx, field, grid, parts.position, a.integrator, a.step_size, horizons)
        entry["fp64_error"] = err
        entry["horizon_99pct_within_1e-3_cells"] = within_horizon(err)
        out[storage] = entry
        field.close()
    return out


def true_rk4(a, ctx, field, grid, parts, p0, r0, stream, steps=3):
    """The same workload with runge_kutta_4_true: four field samples per step
    (the reference's runge_kutta_4 takes one, its system ignoring the state),
    so four times the gathers; throughput and error against the FP64 oracle's
    four-sample RK4."""
    from dpa_b200 import _native as N
    opts = N.AdvectOptions(N.INTEGRATORS["runge_kutta_4_true"], float(np.float32(a.step_size)),
                           0, 0, 0, 1, 0)
    kernel, _, rem, _ = device_steps(ctx, field, opts, p0, r0, stream, steps)
    taken = float((a.iterations - rem.cpu().numpy().astype(np.int64)).sum())
    return {"field_samples_per_step": 4, "kernel_ms": kernel,
            "particle_steps_per_s": taken / (kernel / 1e3),
            "algorithmic_bytes_per_step": 4 * BYTES_PER_STEP[a.storage],
            "fp64_error": fp64_error(ctx, field, grid, parts.position, "runge_kutta_4_true",
                                     a.step_size, (50, 250))}


def systems_forms(a, ctx, grid, parts, p0, r0, pos, rem, term, stream, plain_ms, steps=10):
    """The batched form on the headline workload: field in FP16 (and FP32 for
    comparison), launch parameters (claim, grid, order, block size, particles
    per thread) picked by the autotuner on the same seeds, the order +
    advection sequence replayed from a CUDA graph. Ratios are against this
    run's plain FP32 step (dpa_advect_device, default parameters); the FP16
    entry repeats its FP64-oracle error beside the speed-up."""
    from dpa_b200 import _native as N
    lib = ctx._lib
    out = {}
    saved = N.Tuning()
    ctx.check(lib.dpa_context_get_tuning(ctx.handle, C.byref(saved)))
    for storage in ("f16", "f32"):
        field = ctx.field(grid, storage)
        opts = N.AdvectOptions(N.INTEGRATORS[a.integrator], float(np.float32(a.step_size)),
                               0, 0, 0, 1, 0)
        best = autotune(ctx, field, opts, p0, r0, a.seeds)
        ms = _graph_replays(ctx, field, opts, p0, r0, pos, rem, term, stream, steps)
        taken = float((a.iterations - rem.cpu().numpy().astype(np.int64)).sum())
        out[f"{storage}_autotuned_graph"] = {
            "ms_per_step": ms, "particle_steps_per_s": taken / (ms / 1e3),
            "speedup_vs_plain_f32": plain_ms / ms, "tuning": _tuning_dict(best),
            "fp64_error": fp64_error(ctx, field, grid, parts.position, a.integrator,
                                     a.step_size, (25, 50))}
        ctx.check(lib.dpa_context_set_tuning(ctx.handle, C.byref(saved)))
        field.close()
    return out


# ---------------------------------------------------------------------------
# Configurations beside the headline.

def _pinned(shape, dtype):
    import torch
    t = {np.float32: torch.float32, np.int64: torch.int64, np.uint8: torch.uint8}[dtype]
    return torch.empty(shape, dtype=t, pin_memory=True).numpy()


def _round_call(ctx, field, opts, n, hp, hr, ht, sink):
    from dpa_b200 import _native as N
    ctx.check(ctx._lib.dpa_advect_round(ctx.handle, field.handle, C.byref(opts), n,
                                        hp.ctypes.data_as(C.c_void_p),
                                        hr.ctypes.data_as(C.c_void_p),
                                        ht.ctypes.data_as(C.c_void_p), sink or N.CURVE_SINK(),
                                        None))


def _counting_sink(totals):
    """A curve sink that takes each chunk in place (the curve has crossed to
    the library's pinned host buffers) and counts it."""
    from dpa_b200 import _native as N

    @N.CURVE_SINK
    def sink(user, chunk):
        c = chunk.contents
        totals["vertices"] += c.vertex_count
        totals["indices"] += c.index_count
        totals["chunks"] += 1
        return 0
    return sink


def recording_config(ctx, reps=20, warmup=3, checks=True):
    """The recording configuration (configs[0], the reference's own CPU case):
    ABC flow (A = sqrt 3, B = sqrt 2, C = 1) on 64^3 over [0, 2 pi]^3, 4096
    uniform seeds (seed 0) in the domain, runge_kutta_4 (one field sample per
    step), step 0.01, 1000 iterations, curve recording with uint32 indices and
    angular-velocity colors. A step is one dpa_advect_round with pinned host
    arrays and a sink that takes the curve chunks in place. `value` is the
    round's device work (ordering, advection, curve offsets and emission, from
    the library's events); `e2e` the host call with its copies and syncs."""
    from dpa_b200 import _native as N
    from dpa_b200 import fields, seeds
    lib = ctx._lib
    grid = fields.abc(64)
    offset, size = seeds.seed_box(grid)
    n, iterations, step = 4096, 1000, float(np.float32(0.01))
    pos0 = seeds.generate_random(offset, size, n, iterations,
                                 aabb=([0, 0, 0], [2 * math.pi] * 3), seed=0).position
    field = ctx.field(grid)
    hp, ht = _pinned((n, 3), np.float32), _pinned(n, np.uint8)
    hr = _pinned(n, np.int64).view(np.uint64)
    totals = {"vertices": 0, "indices": 0, "chunks": 0}
    sink = _counting_sink(totals)
    opts = N.AdvectOptions(N.INTEGRATORS["runge_kutta_4"], step, 1, 0, 1, 1, 0)
    ctx.check(lib.dpa_context_set_profiling(ctx.handle, 1))
    launches0 = C.c_uint64()
    walls, device = [], []
    for i in range(warmup + reps):
        hp[:] = pos0
        hr[:] = iterations
        if i == warmup:
            ctx.check(lib.dpa_context_launch_count(ctx.handle, C.byref(launches0)))
        totals.update(vertices=0, indices=0, chunks=0)
        t0 = time.perf_counter()
        _round_call(ctx, field, opts, n, hp, hr, ht, sink)
        wall = time.perf_counter() - t0
        o, k, e = C.c_float(), C.c_float(), C.c_float()
        ctx.check(lib.dpa_context_last_timing(ctx.handle, C.byref(o), C.byref(k)))
        ctx.check(lib.dpa_context_last_emit_timing(ctx.handle, C.byref(e)))
        if i >= warmup:
            walls.append(wall)
            device.append((o.value, k.value, e.value))
    launches1 = C.c_uint64()
    ctx.check(lib.dpa_context_launch_count(ctx.handle, C.byref(launches1)))
    steps_taken = float(np.sum(iterations - hr.astype(np.int64)))
    max_steps = int(np.max(iterations - hr.astype(np.int64)))
    order_ms = statistics.median(d[0] for d in device)
    advect_ms = statistics.median(d[1] for d in device)
    emit_ms = statistics.median(d[2] for d in device)
    device_ms = order_ms + advect_ms + emit_ms
    wall = statistics.median(walls)
    vbytes = totals["vertices"] * 16
    ibytes = totals["indices"] * 4
    out = {
        "workload": "ABC flow 64^3 over [0, 2 pi]^3, 4096 uniform seeds (seed 0), "
                    "runge_kutta_4 (one field sample per step), step 0.01, 1000 iterations, "
                    "recording with uint32 indices and colors",
        "value": steps_taken / (device_ms / 1e3), "unit": UNIT, "ms_per_step": device_ms,
        "particle_steps_per_step": steps_taken, "steps": reps, "warmup": warmup,
        "device_ms": {"order": order_ms, "advect": advect_ms, "emit": emit_ms},
        "e2e": {"value": steps_taken / wall, "unit": UNIT, "ms_per_step": wall * 1e3,
                "h2d_bytes_per_step": n * (12 + 8),
                "d2h_bytes_per_step": n * (12 + 8 + 1) + vbytes + ibytes,
                "call": "dpa_advect_round with pinned host arrays; the curve crosses to the "
                        "library's pinned buffers and the sink takes it in place"},
        "curve": {"vertices": totals["vertices"], "indices": totals["indices"],
                  "chunks": totals["chunks"], "bytes": vbytes + ibytes},
        "gpu_launches_per_step": int(launches1.value - launches0.value) // reps,
        "latency_bound": {
            "longest_particle_steps": max_steps,
            "us_per_step_of_the_longest_particle": advect_ms * 1e3 / max(max_steps, 1),
            "note": "4096 particles fill a fraction of the device; the advection launch lasts as "
                    "long as its longest particle's chain of dependent steps"},
    }
    if checks:
        out["cpu_baseline"] = cpu_rate(grid, "runge_kutta_4", step, pos0,
                                       np.full(n, iterations, np.uint64), 5.0, record=True)
        out["fp64_error"] = fp64_error(ctx, field, grid, pos0, "runge_kutta_4", step,
                                       (50, 100, 250), sample=n)
    field.close()
    return out


def ftle_config(ctx, stream, reps=10, warmup=3, checks=True):
    """The FTLE configuration: ABC flow + 5 % smoothed Gaussian perturbation
    (sigma 3 cells, seed 2) on 256^3 over [0, 2 pi]^3, the 128^3 seed lattice
    (seed_generation_stride 2), runge_kutta_4 (one sample per step), step
    0.02, 250 iterations (T = 5), then the FTLE of the flow map. `value` is
    device-timed lattice advection + FTLE per step; `e2e` the host entry
    points dpa_advect_round + dpa_ftle_estimate with pinned arrays. The FP64
    error is the FTLE against one computed from FP64 oracle trajectories on
    an interior 16^3 block, at the configured T = 5 and at T = 0.5 (25
    steps), where every stencil of the block stays inside the grid."""
    import torch
    from dpa_b200 import _native as N
    from dpa_b200 import fields, seeds
    lib = ctx._lib
    grid = fields.abc_perturbed(256, 0.05, 3.0, 2, device="cuda")
    offset, size = seeds.seed_box(grid)
    lattice = seeds.generate(offset, size, (grid.spacing * np.float32(2)).astype(np.float32),
                             250).position
    n, iterations, step = lattice.shape[0], 250, float(np.float32(0.02))
    # F32 values as edge records (DPA_STORAGE_F32_EDGES): the same bits as F32
    # node storage, one 32-byte load per cell edge for particles that change
    # cells almost every step.
    field = ctx.field(grid, "f32_edges")
    p0 = torch.from_numpy(lattice).cuda()
    r0 = torch.full((n,), iterations, dtype=torch.int64, device="cuda")
    p, r = torch.empty_like(p0), torch.empty_like(r0)
    term = torch.empty(n, dtype=torch.uint8, device="cuda")
    stride = (C.c_float * 3)(2.0, 2.0, 2.0)
    shape = (C.c_uint64 * 3)()
    ftle = torch.empty(128 ** 3, dtype=torch.float32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    opts = N.AdvectOptions(N.INTEGRATORS["runge_kutta_4"], step, 0, 0, 0, 1, 0)
    ctx.check(lib.dpa_context_set_profiling(ctx.handle, 1))

    def one(field_h, horizon=iterations):
        p.copy_(p0)
        r.fill_(horizon)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e2 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.check(lib.dpa_advect_device(ctx.handle, field_h, C.byref(opts), n,
                                        C.c_void_p(p.data_ptr()), C.c_void_p(r.data_ptr()),
                                        C.c_void_p(term.data_ptr()),
                                        C.c_void_p(stream.cuda_stream)))
        e1.record(stream)
        ctx.check(lib.dpa_ftle_estimate_device(
            ctx.handle, field_h, stride, horizon, step, n, C.c_void_p(p0.data_ptr()),
            C.c_void_p(p.data_ptr()), 0, C.c_void_p(ftle.data_ptr()), shape,
            C.c_void_p(stream.cuda_stream)))
        e2.record(stream)
        e2.synchronize()
        o, k = C.c_float(), C.c_float()
        ctx.check(lib.dpa_context_last_timing(ctx.handle, C.byref(o), C.byref(k)))
        return e0.elapsed_time(e2), k.value, e1.elapsed_time(e2)

    for _ in range(warmup):
        flush.fill_(1)
        one(field.handle)
    totals, kernels, ftles = [], [], []
    for i in range(reps):
        flush.fill_(i & 1)
        t, k, f = one(field.handle)
        totals.append(t)
        kernels.append(k)
        ftles.append(f)
    steps_taken = float(np.sum(iterations - r.cpu().numpy()))
    ms = statistics.mean(totals)
    # The same lattice on F32 node storage, for comparison.
    nodes = ctx.field(grid, "f32")
    one(nodes.handle)
    node_kernels = [one(nodes.handle)[1] for _ in range(3)]
    nodes.close()
    # End to end: the host entry points with pinned arrays.
    hp, ht = _pinned((n, 3), np.float32), _pinned(n, np.uint8)
    hr = _pinned(n, np.int64).view(np.uint64)
    hf = _pinned(128 ** 3, np.float32)
    hsh = (C.c_uint64 * 3)()

    def e2e_once():
        hp[:] = lattice
        hr[:] = iterations
        t0 = time.perf_counter()
        _round_call(ctx, field, opts, n, hp, hr, ht, None)
        ctx.check(lib.dpa_ftle_estimate(ctx.handle, field.handle, stride, iterations, step, n,
                                        lattice.ctypes.data_as(C.c_void_p),
                                        hp.ctypes.data_as(C.c_void_p), 0,
                                        hf.ctypes.data_as(C.c_void_p), hsh))
        return time.perf_counter() - t0

    e2e_once()
    e2e = statistics.median([e2e_once() for _ in range(3)])
    out = {
        "workload": "ABC + 5 % smoothed perturbation (sigma 3, seed 2) on 256^3 over "
                    "[0, 2 pi]^3, 128^3 seed lattice (stride 2), runge_kutta_4, step 0.02, "
                    "250 iterations, then FTLE (FP64 eigenvalue and log)",
        "storage": "f32_edges (F32 values as one 32-byte record per cell edge; results "
                   "identical to f32 node storage)",
        "value": steps_taken / (ms / 1e3), "unit": UNIT, "ms_per_step": ms,
        "particle_steps_per_step": steps_taken, "steps": reps, "warmup": warmup,
        "kernel_ms": statistics.mean(kernels), "ftle_ms": statistics.mean(ftles),
        "kernel_ms_f32_node_storage": statistics.mean(node_kernels),
        "e2e": {"value": steps_taken / e2e, "unit": UNIT, "ms_per_step": e2e * 1e3,
                "h2d_bytes_per_step": n * (12 + 8) + n * 24,
                "d2h_bytes_per_step": n * (12 + 8 + 1) + 128 ** 3 * 4,
                "call": "dpa_advect_round + dpa_ftle_estimate with pinned host arrays"},
        "roofline": roofline(statistics.mean(kernels) / 1e3, steps_taken, n, "f32",
                             "ftle_lattice_f32_edges", gather_peaks(ctx)),
    }
    if not checks:
        field.close()
        return out
    # FTLE of both storages against the FP64 oracle, at T = 5 and T = 0.5.
    err = {}
    for horizon in (iterations, 25):
        got = {}
        for storage in ("f32", "f16"):
            f = field if storage == "f32" else ctx.field(grid, storage)
            one(f.handle, horizon)
            got[storage] = ftle.cpu().numpy()
            if f is not field:
                f.close()
        err[f"steps_{horizon}"] = ftle_fp64_error(grid, lattice, got, horizon, step)
    out["ftle_fp64_error"] = err
    sample = lattice[np.sort(np.random.default_rng(11).choice(n, 200_000, False))]
    out["cpu_baseline"] = cpu_rate(grid, "runge_kutta_4", step, sample,
                                   np.full(sample.shape[0], iterations, np.uint64), 8.0,
                                   describe=", a seeded random sample of the lattice")
    field.close()
    return out


def ftle_fp64_error(grid, lattice, ftle_by_storage, iterations, step, lo=60, m=16):
    """FTLE error against the FP64 oracle on an m^3 block of interior lattice
    cells starting at lattice index lo (clear of the planes where the
    reference's cell mapping collides): the block and a one-cell halo are
    advected in double (the reference's one-sample RK4), the flow-map
    Jacobian is taken by central differences over the lattice spacing, and
    FTLE = ln sqrt(lambda_max(J^T J)) / |step * iterations|. Returns the
    relative error of each storage's GPU FTLE over the block, over all its
    cells and over the cells whose whole stencil ran every iteration inside
    the grid (elsewhere the flow map holds exit positions, which a one-step
    difference in the exit moves by a cell or more)."""
    ob = _oracle()
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
    Cm = np.einsum("...ki,...kj->...ij", J, J)
    lam = np.linalg.eigvalsh(Cm)[..., -1]
    want = np.log(np.sqrt(lam)) / abs(float(np.float32(step) * np.float32(iterations)))
    done = (r.termination == 0).reshape(m + 2, m + 2, m + 2)
    inside = done[1:-1, 1:-1, 1:-1].copy()
    for sl in [(slice(2, None), slice(1, -1), slice(1, -1)),
               (slice(None, -2), slice(1, -1), slice(1, -1)),
               (slice(1, -1), slice(2, None), slice(1, -1)),
               (slice(1, -1), slice(None, -2), slice(1, -1)),
               (slice(1, -1), slice(1, -1), slice(2, None)),
               (slice(1, -1), slice(1, -1), slice(None, -2))]:
        inside &= done[sl]
    out = {"block": f"lattice cells [{lo}, {lo + m})^3 of 128^3, FP64 reference-semantics RK4, "
                    f"{iterations} steps"}
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
                           "p99_rel": float(np.percentile(rel, 99)), "max_rel": float(rel.max()),
                           "within_1e-3_rel": float(np.mean(rel <= 1e-3))}
        out[storage] = entry
    return out


def batch_sets(n_grid, total, sets=64, seed=3):
    """64 seed sets: sizes log-uniform in [1e3, 1e6], then scaled so that they
    sum to `total` (the configuration's 16 M; a plain log-uniform draw of 64
    sets averages 9.3 M), iterations uniform in [200, 4000]."""
    rng = np.random.default_rng(seed)
    raw = np.exp(rng.uniform(np.log(1e3), np.log(1e6), size=sets))
    sizes = np.maximum(np.floor(raw * total / raw.sum()).astype(np.int64), 1)
    sizes[-1] += total - int(sizes.sum())
    iters = rng.integers(200, 4001, size=sets)
    return sizes, iters


def batched_config(ctx, stream, a, reps=2):
    """The large batched configuration: a curl-noise field of 512^3 (sigma 8,
    seed 3; 2.1 GB F32 / 1.1 GB F16 repacked), 64 seed sets of log-uniform
    sizes scaled to 16,777,216 particles in all, iterations uniform in
    [200, 4000] per set, runge_kutta_4 step 0.25.
      device: the batch in one persistent launch replayed from a CUDA graph
              with autotuned launch parameters, F32 and F16 fields, beside one
              plain FP32 dpa_advect_device call over the same particles;
      e2e:    the batch as one recording round through dpa_advect_round from
              pinned host arrays: curves pruned, indexed and colored, uint64
              indices (particles per round x iterations > 2^32 - 1, the rule of
              pipeline.cpp:155), streamed to the host in pieces through a sink
              that takes them in place -- bound by the host link, whose pinned
              device-to-host bandwidth is measured beside it."""
    import torch
    from dpa_b200 import _native as N
    from dpa_b200 import fields, seeds
    lib = ctx._lib
    ctx.check(lib.dpa_context_set_profiling(ctx.handle, 1))
    n_grid = a.batch_n
    grid = fields.curl_noise(n_grid, 8.0, 3, device="cuda")
    torch.cuda.empty_cache()
    total = a.batch_particles if n_grid == 512 else int(a.batch_particles * (n_grid / 512) ** 3)
    sizes, iters = batch_sets(n_grid, total)
    offset, size = seeds.seed_box(grid)
    box = ([0.0] * 3, [float(n_grid - 1)] * 3)
    pos_h = seeds.generate_random(offset, size, total, 0, aabb=box, seed=3).position
    rem_h = np.repeat(iters, sizes).astype(np.int64)
    set_offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint64)
    step = float(np.float32(0.25))
    out = {"workload": f"curl noise {n_grid}^3 (sigma 8, seed 3), 64 seed sets, sizes "
                       f"log-uniform in [1e3, 1e6] scaled to {total} particles (largest "
                       f"{int(sizes.max())}), iterations uniform in [200, 4000], runge_kutta_4 "
                       "step 0.25",
           "sets": 64, "particles": total,
           "set_sizes": {"min": int(sizes.min()), "max": int(sizes.max())},
           "iterations": {"min": int(iters.min()), "max": int(iters.max())}}
    p0 = torch.from_numpy(pos_h).cuda()
    r0 = torch.from_numpy(rem_h).cuda()
    pos, rem = torch.empty_like(p0), torch.empty_like(r0)
    term = torch.empty(total, dtype=torch.uint8, device="cuda")
    saved = N.Tuning()
    ctx.check(lib.dpa_context_get_tuning(ctx.handle, C.byref(saved)))
    steps_total = None
    for storage in ("f32", "f16"):
        field = ctx.field(grid, storage)
        opts = N.AdvectOptions(N.INTEGRATORS["runge_kutta_4"], step, 0, 0, 0, 1, 0)
        if storage == "f32":
            plain, _, prem, _ = device_steps(ctx, field, opts, p0, r0, stream, reps)
            steps_total = float((r0 - prem).sum().item())
            out["plain_f32"] = {"ms": plain, "particle_steps_per_s": steps_total / (plain / 1e3),
                                "call": "one dpa_advect_device over all particles, default "
                                        "launch parameters"}
        best = autotune(ctx, field, opts, p0, r0, total, sample_steps=400)
        ms = _graph_replays(ctx, field, opts, p0, r0, pos, rem, term, stream, reps)
        taken = float((r0 - rem).sum().item())
        set_steps = np.zeros(64, np.uint64)
        pos.copy_(p0)
        rem.copy_(r0)
        ctx.check(lib.dpa_advect_batch_device(
            ctx.handle, field.handle, C.byref(opts), 64, set_offsets.ctypes.data_as(N._U64P),
            C.c_void_p(pos.data_ptr()), C.c_void_p(rem.data_ptr()), C.c_void_p(term.data_ptr()),
            set_steps.ctypes.data_as(N._U64P), C.c_void_p(stream.cuda_stream)))
        out[storage] = {"ms_per_batch": ms, "particle_steps": taken,
                        "particle_steps_per_s": taken / (ms / 1e3), "tuning": _tuning_dict(best),
                        "set_steps_sum_matches": bool(int(set_steps.sum()) == int(taken)),
                        "field_device_bytes": field.device_bytes,
                        "fp64_error": fp64_error(ctx, field, grid, pos_h, "runge_kutta_4", step,
                                                 (25, 50, 250))}
        ctx.check(lib.dpa_context_set_tuning(ctx.handle, C.byref(saved)))
        if storage == "f32":
            out["value"] = taken / (ms / 1e3)
            out["unit"] = UNIT
            out["ms_per_step"] = ms
            out["cpu_baseline"] = cpu_rate(grid, "runge_kutta_4", step, pos_h, rem_h.astype(
                np.uint64), 8.0, record=True, max_count=16384,
                describe=", the batch's first seeds with their set's iterations")
            # End to end with recording, streamed.
            ctx.set_staging_limit(8 << 30)
            hp, ht = _pinned((total, 3), np.float32), _pinned(total, np.uint8)
            hr = _pinned(total, np.int64).view(np.uint64)
            totals = {"vertices": 0, "indices": 0, "chunks": 0}
            sink = _counting_sink(totals)
            ropts = N.AdvectOptions(N.INTEGRATORS["runge_kutta_4"], step, 1, 1, 1, 1, 0)
            hp[:] = pos_h
            hr[:] = rem_h.astype(np.uint64)
            t0 = time.perf_counter()
            _round_call(ctx, field, ropts, total, hp, hr, ht, sink)
            wall = time.perf_counter() - t0
            rec_steps = float(np.sum(rem_h.astype(np.int64) - hr.astype(np.int64)))
            curve_bytes = totals["vertices"] * 16 + totals["indices"] * 8
            out["e2e"] = {"value": rec_steps / wall, "unit": UNIT, "seconds": wall,
                          "h2d_bytes_per_step": total * (12 + 8),
                          "d2h_bytes_per_step": total * (12 + 8 + 1) + curve_bytes,
                          "curve_vertices": totals["vertices"], "indices": totals["indices"],
                          "index_width": "uint64", "chunks": totals["chunks"],
                          "curve_GB": curve_bytes / 1e9, "curve_GB_per_s": curve_bytes / 1e9 / wall,
                          "host_link_d2h_GB_per_s": d2h_bandwidth(),
                          "steps_match_device_run": bool(rec_steps == taken),
                          "call": "dpa_advect_round over the whole batch with recording, "
                                  "colors and uint64 indices, pinned host arrays, staging "
                                  "limit 8 GiB"}
            del hp, hr, ht
            ctx.set_staging_limit(1 << 30)
        field.close()
    out["f16_batched_vs_plain_f32"] = out["plain_f32"]["ms"] / out["f16"]["ms_per_batch"]
    del p0, r0, pos, rem, term
    torch.cuda.empty_cache()
    return out


def d2h_bandwidth(nbytes=1 << 30):
    """Pinned device-to-host copy bandwidth (GB/s) of this box, one 1 GiB copy."""
    import torch
    src = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    dst = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    dst.copy_(src, non_blocking=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    dst.copy_(src, non_blocking=True)
    torch.cuda.synchronize()
    return nbytes / 1e9 / (time.perf_counter() - t0)


def serving_run(a, ctx, arrival_seed=4, storage="f16", probe=False):
    """The serving configuration: resident 256^3 and 512^3 curl-noise fields
    (sigma 4 / seed 1 and sigma 8 / seed 3) and the double gyre on
    128 x 64 x 64 with 32 time slices, stored in `storage` (the FP16 served
    form by default); Poisson arrivals (seed `arrival_seed`) at 200
    requests/s for serve_seconds. Request mix: 10 % FTLE on a 64^3 lattice of
    the 256^3 field; 30 % pathlines through the gyre (start times uniform in
    [0, 5], step 0.002); 60 % on either curl-noise field. Five in nine of the
    pathline and curl-noise requests record curves (half of all requests).
    Seeds are log-uniform in [1e2, 1e6], except for recording requests, whose
    seeds are log-uniform in [1e2, 2e4]: the configured mix's recording
    requests (up to 1e6 seeds x 5000 steps) return about 4 GB of curve each,
    some 400 GB/s at 100 such requests per second, eight times what the host
    link carries, so their queue would grow without bound; at 2e4 seeds the
    curves need about a quarter of the link. Iterations uniform in [100,
    5000]. Admission passes small requests (at most 65,536 seeds) past large
    ones that wait for room, keeps 10 % of the 12 M slots for them and lets
    the oldest request be passed by large ones for at most 250 ms (small ones
    keep passing it within that 10 %). Latency is submit to result;
    throughput counts particle-steps over the wall time of the run. Results
    are returned in an 8 GiB pinned arena and dropped once their times are
    read (no copy), except (probe) for a few
    end-position requests of 512 seeds x 50 steps on the 256^3 field, whose
    positions are compared with the FP64 oracle."""
    import threading as th
    from dpa_b200 import fields, seeds
    from dpa_b200.serve import Server
    grid = fields.curl_noise(256, 4.0, 1, device="cuda")
    big = fields.curl_noise(512, 8.0, 3, device="cuda")
    gyre = fields.double_gyre()
    resident = [ctx.field(grid, storage), ctx.field(big, storage), ctx.field(gyre, storage)]
    rng = np.random.default_rng(arrival_seed)
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
    plan = []  # (time, field index, seeds, iterations, record, ftle, start time, step, probe)
    t = 0.0
    while True:
        t += rng.exponential(1.0 / 200.0)
        if t > a.serve_seconds:
            break
        kind = rng.random()
        iters = int(rng.integers(100, 5001))
        if kind < 0.1:
            plan.append((t, 0, lattice, iters, False, True, 0.0, a.step_size, False))
            continue
        record = rng.random() < 5.0 / 9.0
        hi = 2e4 if record else 1e6
        count = int(np.exp(rng.uniform(np.log(1e2), np.log(hi))))
        if kind < 0.4:
            start = int(rng.integers(0, len(gyre_pool) - count))
            plan.append((t, 2, gyre_pool[start:start + count], iters, record, False,
                         float(rng.uniform(0.0, 5.0)), 0.002, False))
            continue
        which = int(rng.integers(0, 2))
        start = int(rng.integers(0, len(pools[which]) - count))
        plan.append((t, which, pools[which][start:start + count], iters, record, False, 0.0,
                     a.step_size, False))
    if probe:  # eight small end-position requests spread over the run
        for k in range(8):
            when = a.serve_seconds * (k + 0.5) / 8
            plan.append((when, 0, pools[0][k * 512:(k + 1) * 512], 50, False, False, 0.0,
                         a.step_size, True))
        plan.sort(key=lambda p: p[0])
    results = []
    probes = {}
    with Server(ctx, particle_capacity=12_000_000, vertex_capacity=1_200_000_000,
                steps_per_tick=64, max_requests=1024, small_request_seeds=65536,
                reserved_percent=10, max_bypass_ms=250, response_bytes=8 << 30) as server:
        fids = [server.add_field(f) for f in resident]
        done = th.Event()
        probe_ids = set()

        def collect():
            while len(results) < len(plan):
                r = server.poll(wait_ms=50, copy_ids=probe_ids)
                if r is not None:
                    # Keep the times, drop the arrays (a run of recording
                    # requests returns tens of GB of curves).
                    results.append(types.SimpleNamespace(
                        id=r.id, latency=r.latency, queued=r.queued, admitted=r.admitted,
                        finished=r.finished, particle_steps=r.particle_steps, status=r.status))
                    if r.id in probe_ids:
                        probes[r.id] = r
                elif done.is_set() and server.stats()["completed"] >= len(plan) and \
                        len(results) >= len(plan):
                    break
        poller = th.Thread(target=collect, daemon=True)
        poller.start()
        t0 = time.perf_counter()
        for when, which, pos, iters, record, ftle, start_time, step, is_probe in plan:
            delay = when - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            rid = server.submit(fids[which], pos, iters, a.integrator, step, record=record,
                                ftle=ftle, seed_stride=(4.0, 4.0, 4.0), start_time=start_time)
            if is_probe:
                probe_ids.add(rid)
        done.set()
        poller.join(timeout=600)
        wall = time.perf_counter() - t0
        stats = server.stats()
    lat = np.array([r.latency for r in results]) * 1e3
    steps = float(sum(r.particle_steps for r in results))
    kinds = {"ftle": sum(1 for p in plan if p[5]), "recording": sum(1 for p in plan if p[4]),
             "pathlines": sum(1 for p in plan if p[1] == 2),
             "on_512": sum(1 for p in plan if p[1] == 1)}

    def pct(values):
        v = np.asarray(values, np.float64) * 1e3
        return {"p50": float(np.percentile(v, 50)), "p99": float(np.percentile(v, 99))} \
            if len(v) else None

    kind_of = {}
    for i, p in enumerate(plan):
        kind_of[i + 1] = ("probe" if p[8] else "ftle" if p[5] else "pathlines" if p[1] == 2
                          else "recording" if p[4] else "end_positions")
    by_kind = {}
    for k in ("end_positions", "recording", "pathlines", "ftle"):
        rs = [r for r in results if kind_of.get(r.id) == k]
        by_kind[k] = {"latency_ms": pct([r.latency for r in rs]),
                      "queue_wait_ms": pct([r.admitted - r.queued for r in rs]),
                      "service_ms": pct([r.finished - r.admitted for r in rs])}
    out = {"arrival_seed": arrival_seed, "requests": len(plan), "completed": len(results),
           "failed": sum(1 for r in results if r.status != 0),
           "wall_seconds": wall,
           "_latencies_ms": lat,  # pooled over the runs by serving_config, then dropped
           "latency_ms": {"p50": float(np.percentile(lat, 50)),
                          "p99": float(np.percentile(lat, 99)), "max": float(lat.max())},
           "queue_wait_ms": pct([r.admitted - r.queued for r in results]),
           "by_kind": by_kind,
           "particle_steps_per_s": steps / wall, "ticks": int(stats["ticks"]),
           "launches": int(stats["launches"]), "busy_seconds": float(stats["busy_seconds"]),
           "tick_device_seconds": float(stats["tick_device_seconds"]),
           "admission": {k: stats[k] for k in ("peak_slots", "peak_vertices", "slot_refusals",
                                                "vertex_refusals", "overdue_scans",
                                                "peak_finishing", "finish_seconds")},
           "mix": kinds}
    if probe and probes:
        ob = _oracle()
        og = ob.OracleGrid.of(grid)
        errs = []
        for rid, r in probes.items():
            pos = plan[rid - 1][2]  # ids follow submission order from 1
            ref = ob.advect64(og, a.integrator, a.step_size, pos, np.full(len(pos), 50, np.uint64))
            gpu = types.SimpleNamespace(position=r.positions, termination=r.termination)
            errs.append(position_error(gpu, ref, 1.0))
        out["fp64_error_served"] = {
            "requests": len(errs), "steps": 50,
            "median_cells": statistics.median(e["median_cells"] for e in errs if e["median_cells"]
                                              is not None),
            "max_cells": max(e["max_cells"] for e in errs if e["max_cells"] is not None),
            "within_1e-3_cells": statistics.mean(e["within_1e-3_cells"] for e in errs
                                                 if e["within_1e-3_cells"] is not None)}
    for f in resident:
        f.close()
    return out


def serving_config(a, ctx):
    runs = [serving_run(a, ctx, arrival_seed=4 + i, probe=(i == 0)) for i in range(a.serve_runs)]
    p99 = [r["latency_ms"]["p99"] for r in runs]
    p50 = [r["latency_ms"]["p50"] for r in runs]
    # One 20 s run holds ~4,000 requests, so its p99 rests on its ~40 slowest;
    # the pooled figures take every request of every run.
    pooled = np.concatenate([r.pop("_latencies_ms") for r in runs])
    return {"rate_per_s": 200.0, "seconds_of_arrivals_per_run": a.serve_seconds,
            "field_storage": "f16", "runs": runs,
            "latency_ms": {"p50_median": statistics.median(p50), "p99_median": statistics.median(p99),
                           "p99_min": min(p99), "p99_max": max(p99),
                           "p99_spread": max(p99) / max(min(p99), 1e-9),
                           "p50_pooled": float(np.percentile(pooled, 50)),
                           "p99_pooled": float(np.percentile(pooled, 99)),
                           "requests_pooled": int(pooled.size)},
            "particle_steps_per_s": statistics.mean(r["particle_steps_per_s"] for r in runs),
            "fp64_error_served": runs[0].get("fp64_error_served")}


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


def run_one(a):
    """One configuration alone (--workload recording / ftle / batched / serving)."""
    import torch
    import dpa_b200
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    ctx = dpa_b200.Context(int(os.environ.get("LOCAL_RANK", "0")))
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    checks = not a.no_cpu_baseline  # the CPU baseline and the FP64-oracle errors
    if a.workload == "recording":
        out = recording_config(ctx, checks=checks)
    elif a.workload == "ftle":
        out = ftle_config(ctx, stream, checks=checks)
    elif a.workload == "batched":
        out = batched_config(ctx, stream, a)
    else:
        out = serving_config(a, ctx)
    out.update({"metric": METRIC, "n_gpus": 1, "higher_is_better": True, "dtype": "f32",
                "data": "synthetic", "config": {"workload": a.workload}})
    print(json.dumps(out), flush=True)
    ctx.close()
    return 0


def run_gpu(a):
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
    opts = N.AdvectOptions(N.INTEGRATORS[a.integrator], float(np.float32(a.step_size)), 0, 0, 0, 1,
                           0)
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
    time.sleep(0.5)  # nvidia-smi's first readings
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t_begin = time.perf_counter()
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
    t_end = time.perf_counter()
    time.sleep(0.1)
    clock_info = clocks.stop((t_begin, t_end))
    launches1 = C.c_uint64()
    ctx.check(lib.dpa_context_launch_count(ctx.handle, C.byref(launches1)))
    gpu_launches = int(launches1.value - launches0.value)

    rem_out = rem.cpu().numpy().astype(np.int64)
    steps_taken = float(np.sum(a.iterations - rem_out))
    ms_per_step = total_ms / a.steps
    ms_max, steps_total = combine_over_ranks(ms_per_step, steps_taken, "cuda")
    value = steps_total / (ms_max / 1e3)

    # End to end through the host C ABI with pinned host buffers.
    host_pos = torch.empty((n, 3), dtype=torch.float32, pin_memory=True).numpy()
    host_rem = torch.empty(n, dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
    host_term = torch.empty(n, dtype=torch.uint8, pin_memory=True).numpy()
    e2e_steps = max(1, min(a.steps, 3))

    def e2e_once():
        host_pos[:] = parts.position
        host_rem[:] = a.iterations
        t0 = time.perf_counter()
        ctx.check(lib.dpa_advect_round(ctx.handle, field.handle, C.byref(opts), n,
                                       host_pos.ctypes.data_as(C.c_void_p),
                                       host_rem.ctypes.data_as(C.c_void_p),
                                       host_term.ctypes.data_as(C.c_void_p), N.CURVE_SINK(), None))
        return time.perf_counter() - t0

    e2e_once()
    e2e_times = [e2e_once() for _ in range(e2e_steps)]
    e2e_steps_taken = float(np.sum(a.iterations - host_rem.astype(np.int64)))
    e2e_max, e2e_total = combine_over_ranks(statistics.mean(e2e_times), e2e_steps_taken, "cuda")
    e2e_value = e2e_total / e2e_max

    kernel_s = statistics.mean(kernel_ms) / 1e3
    peaks = gather_peaks(ctx)
    key = f"throughput_{a.storage}_{a.integrator}_n{a.n}"
    default_workload = a.seeds == 1 << 20 and a.iterations == 2000 and a.step_size == 0.25
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(a, world),
        "particle_steps_per_step": steps_total,
        "kernel_ms": statistics.mean(kernel_ms), "order_ms": statistics.mean(order_ms),
        "roofline": roofline(kernel_s, steps_taken, n, a.storage,
                             key if default_workload else "none", peaks),
        "gather_peaks_gbs": peaks,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": n * (12 + 8),
                "d2h_bytes_per_step": n * (12 + 8 + 1),
                "call": "dpa_advect_round with pinned host buffers (wall clock around the "
                        "synchronous call)"},
        "gpu_launches": gpu_launches,
        "clocks": clock_info,
    }
    tuning = N.Tuning()
    ctx.check(lib.dpa_context_get_tuning(ctx.handle, C.byref(tuning)))
    out["tuning"] = _tuning_dict(tuning)
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(a, grid, parts, a.cpu_seconds)
        out["precision_forms"] = precision_forms(a, ctx, grid, parts, pristine_pos, pristine_rem,
                                                 stream, statistics.mean(kernel_ms))
        out["fp64_error"] = out["precision_forms"][a.storage]["fp64_error"]
        out["true_rk4"] = true_rk4(a, ctx, field, grid, parts, pristine_pos, pristine_rem, stream)
        if not a.no_systems:
            out["systems_forms"] = systems_forms(a, ctx, grid, parts, pristine_pos, pristine_rem,
                                                 pos, rem, term, stream, ms_max)
            field.close()
            field = None
            del pristine_pos, pristine_rem, pos, rem, term, flush
            torch.cuda.empty_cache()
            out["recording"] = recording_config(ctx)
            out["ftle"] = ftle_config(ctx, stream)
            torch.cuda.empty_cache()
            out["batched"] = batched_config(ctx, stream, a)
            out["serving"] = serving_config(a, ctx)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if field is not None:
        field.close()
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    a = parse_args()
    if a.impl == "reference":
        return run_reference(a)
    if a.workload != "throughput":
        return run_one(a)
    return run_gpu(a)


if __name__ == "__main__":
    sys.exit(main())
