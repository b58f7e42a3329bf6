#!/usr/bin/env python
"""Benchmark of the B200 Yee-FDTD engine.

Headline (one bench "step" = one whole FDTD job): 2D TM, 4000 x 1500 cells at
dx = 10 nm with 20-cell CPML, a seeded Bernoulli Si/SiO2 pixel design region
in an SOI waveguide, TM0 mode source, 101-wavelength DFT monitors over
1.5-1.6 um, 30000 time steps, FP32 fields with Kahan-compensated FP32 DFT
sums.  The fields (2 x 72 MB ping-pong + 12 MB material index) exceed the
126 MB L2, so no flush is needed between timed steps.  The line states the
result's error against an FP64 run of the same job (error_vs_fp64); the FP64
form itself is held to the FP64 oracle at this grid size by the GPU tests.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload pixel2d|coupler|pillar3d|coupler_batch|serve|fdfd] [--no-forms]

At N = 1 the headline line also carries one sub-record per other form of
the engine, each with its own timing, clocks and roofline:
  c1_coupler_fp64   800 x 300 FP64 TE grating coupler, 8000 steps (the plain form)
  c3_pillar_fp32 / c3_pillar_fp64
                    3D TiO2 pillar lattice, 600 x 600 x 300, 1000 of its 6000 steps
  c4_coupler_batch  256 uneven FP32 grating couplers, 10000 steps, one batched call
  c5_served         a Poisson stream of 100 mixed 2D / 3D FP32 jobs at 80 % of the
                    measured capacity through the serving loop (p50 / p99 latency)
  fdfd2d            the 2D TE frequency-domain solver on a 501 x 221 SOI slab:
                    factorisation, solve and adjoint solve times, error vs the oracle
--workload runs one of them alone as its own line.

Under torchrun every rank runs its own replica of the job on its GPU (a
single job fits one GPU: "replicas only", weak scaling); rank 0 prints one
JSON line with the whole-job aggregate.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
import warnings

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "Yee Mcells/s"
UNIT = "Mcell-updates/s"
BYTES_PER_CELL_UPDATE = {("TM", "single"): 26, ("TM", "double"): 50, ("TE", "single"): 25, ("TE", "double"): 49}
BYTES_3D = {"single": 51, "double": 99}
PIXEL2D_WORKLOAD = ("2D TM pixel region 4000x1500 dx=10nm 20-cell CPML, TM0 source, "
                    "101-lambda DFT (3 x-lines, 2 z-lines), 30000 time steps per job")
PIXEL2D_DATA = "synthetic (seeded Bernoulli Si/SiO2 pixel map, 4000x1500)"


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="single", choices=["single", "double"])
    ap.add_argument("--time-steps", type=int, default=0, help="FDTD time steps per job (0: the workload's own)")
    ap.add_argument("--cpu-sample-steps", type=int, default=300)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="headline only, without the sub-records")
    ap.add_argument("--workload", default="pixel2d", choices=["pixel2d", "coupler", "pillar3d", "pillar3d_slabs", "coupler_batch", "serve",
                                                       "fdfd"],
                    help="pixel2d is the headline; the others measure one form alone")
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--size3d", default="600,600,300", help="pillar3d grid NX,NY,NZ (smaller for profiling)")
    ap.add_argument("--slabs", type=int, default=2, help="pillar3d_slabs: z slabs of the grid")
    ap.add_argument("--serve-jobs", type=int, default=100)
    ap.add_argument("--serve-load", type=float, default=0.8, help="arrival rate as a fraction of the measured capacity")
    ap.add_argument("--serve-rate", type=float, default=0.0, help="fixed arrival rate (jobs/s) instead of --serve-load")
    ap.add_argument("--serve-capacity-jobs", type=int, default=24)
    ap.add_argument("--serve-max-cells", type=float, default=5e7)
    ap.add_argument("--serve-macro", type=int, default=150)
    ap.add_argument("--serve-check-frac", type=float, default=0.25)
    return ap.parse_args(argv)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


def measured_peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic_per_cell_update(name="interior_kernel_tm_pixel_4000x1500.json"):
    """DRAM bytes per cell update of a kernel from its committed ncu summary
    (one capture; scaled here to the cell updates of a launch)."""
    p = os.path.join(HERE, "profiles", name)
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["dram_bytes_per_cell_update"])
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"orf_clocks_{os.getpid()}_{index}_{time.monotonic_ns()}.csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}",
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines()]
            os.remove(self.path)
        except Exception:
            return None
        sm = [float(r[0]) for r in rows if r and r[0].strip().replace(".", "").isdigit()]
        if not sm:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for n, v in zip(names, r[4:8]):
                if v.strip() == "Active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][1]), "samples": len(sm),
                "reasons": sorted(reasons)}


def cpu_sample(sim, sample_steps):
    """The oracle (C++ restatement, FP32 fields as the GPU form) on all host
    cores, over the first sample_steps time steps of the headline job."""
    import oracle
    s = dict(sim)
    S = 0.99 / math.sqrt(2) * 0.01
    s["maxTime"] = sample_steps * S
    threads = os.cpu_count() or 1
    t = time.perf_counter()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        oracle.fdtd2D(s, threads=threads)
    dt = time.perf_counter() - t
    cells = s["epsX"].shape[0] * (s["epsZ"].shape[1])
    return {"value": cells * sample_steps / dt / 1e6, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"TM pixel-region grid {cells} cells, {sample_steps} of 30000 time steps, "
                      f"{s['precision']} fields"}, dt


def run_reference(args):
    """The reference's CPU path for this workload: MATLAB P-code, which cannot
    run here; the oracle port (same equations) on all host cores, each step a
    bounded sample of the headline job (the cpu_baseline sample)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from opticrcwafdtd_b200 import workloads
    sim = workloads.pixel_region_sim(precision=args.precision)
    vals = []
    secs = []
    r = None
    for i in range(args.warmup + args.steps):
        r, dt = cpu_sample(sim, args.cpu_sample_steps)
        if i >= args.warmup:
            vals.append(r["value"])
            secs.append(dt)
    v = statistics.mean(vals)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(secs), "higher_is_better": True,
        "dtype": "f32" if args.precision == "single" else "f64", "data": PIXEL2D_DATA,
        "config": {"workload": PIXEL2D_WORKLOAD, "sample": r["sample"]},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": r["cores"], "kind": "port", "sample": r["sample"]},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference (MATLAB P-code) cannot run on this box; CPU oracle restatement timed instead",
    }), flush=True)


def _init_dist(local, world):
    import torch
    torch.cuda.set_device(local)
    if world <= 1:
        return None
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    return dist


def _max_over_ranks(dist, v):
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(dist):
    if dist is not None:
        dist.barrier()


def _roofline(st, bpc, kernel, kind="interior"):
    """Roofline of a step kernel from its per-launch CUDA events."""
    peak, peak_kind = measured_peaks()
    ms, launches, cu = st[f"{kind}_ms"], st[f"{kind}_launches"], st[f"{kind}_cell_updates"]
    if ms <= 0 or launches <= 0:
        return None
    per_launch_bytes = bpc * cu / launches
    launch_s = ms / 1e3 / launches
    achieved = per_launch_bytes / launch_s / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
            "traffic": None, "kernel": kernel, "algorithmic_bytes_per_cell_update": bpc,
            "cell_updates_per_launch": cu / launches, "avg_launch_ms": launch_s * 1e3}


def _whole_frac(cell_updates_per_s, bpc):
    peak, kind = measured_peaks()
    a = cell_updates_per_s * bpc / 1e9
    return {"achieved_gbs": a, "peak": peak, "frac": a / peak, "of": kind,
            "algorithmic_bytes_per_cell_update": bpc}


def _line_errors(a, b, inc):
    """Error of result a against result b (the FP64 form): largest DFT-line
    difference over that line's largest magnitude, and the largest absolute
    difference of the transmissions T = flux / inc."""
    import numpy as np
    line = 0.0
    for k in ("P", "B", "PZ", "AZ"):
        if b[k].size:
            line = max(line, float(np.max(np.abs(a[k] - b[k])) / max(1e-300, np.max(np.abs(b[k])))))
    tr = 0.0
    for k in ("flux", "fluxZ"):
        if b[k].size:
            tr = max(tr, float(np.max(np.abs(a[k] / inc - b[k] / inc))))
    return line, tr


def bench_pixel2d(args, rank, world, local, dist):
    """Headline: whole 2D TM pixel-region jobs, device-resident inputs
    (--workload coupler: the 800 x 300 FP64 TE grating coupler instead)."""
    import numpy as np
    import torch
    from opticrcwafdtd_b200 import Context, Job, fdtd2D, workloads

    coupler = args.workload == "coupler"
    if coupler:
        nsteps = args.time_steps or 8000
        args.precision = "double"
        sim = workloads.coupler_sim(precision="double", steps=nsteps)
        pol, nx, nz = "TE", sim["eps"].shape[0], sim["eps"].shape[1]
        data = "synthetic (SOI grating coupler: 20 x 630 nm periods, ff 0.5, 70 nm etch)"
        wl = ("2D TE SOI grating coupler 800x300 dx=20nm 20-cell CPML, TE0 source, 51-lambda DFT, "
              f"{nsteps} time steps per job, FP64")
        l2 = "working set below L2 (this small case runs from L2)"
    else:
        nsteps = args.time_steps or 30000
        sim = workloads.pixel_region_sim(precision=args.precision, steps=nsteps)
        pol, nx, nz = "TM", sim["epsX"].shape[0], sim["epsZ"].shape[1]
        data = PIXEL2D_DATA
        wl = PIXEL2D_WORKLOAD if nsteps == 30000 else PIXEL2D_WORKLOAD.replace("30000", str(nsteps))
        l2 = "inputs larger than L2 (156 MB working set > 126 MB)"
    cells = nx * nz
    stream = torch.cuda.current_stream()
    ctx = Context(local, stream=stream.cuda_stream)
    job = Job(sim, ctx)

    def one_job():
        job.reset()
        job.advance(nsteps)

    for _ in range(args.warmup):
        one_job()
    # timed region: the production path (chunk sequence replayed as CUDA graphs)
    _barrier(dist)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            one_job()
        ev1.record(stream)
        torch.cuda.synchronize()
    _barrier(dist)
    ms = _max_over_ranks(dist, ev0.elapsed_time(ev1))
    value = cells * nsteps * args.steps * world / (ms / 1e3) / 1e6

    # one more job with CUDA events around every launch (graphs off): per-kernel
    # durations for the roofline and the launch count
    ctx.reset_stats()
    ctx.set_timing(True)
    one_job()
    torch.cuda.synchronize()
    st = ctx.stats()
    ctx.set_timing(False)
    launches_per_job = st["interior_launches"] + st["frame_launches"] + st["flush_launches"]
    bpc = BYTES_PER_CELL_UPDATE[(pol, args.precision)]
    roof = _roofline(st, bpc, "k_step2d_fast (interior tiles, PML=false)")
    if roof:
        if not coupler:
            tpc = ncu_traffic_per_cell_update()
            roof["traffic"] = tpc * roof["cell_updates_per_launch"] if tpc else None
        roof["share_of_step_kernels"] = st["interior_ms"] / max(1e-9, st["interior_ms"] + st["frame_ms"])
        roof["frame_kernel_avg_launch_ms"] = st["frame_ms"] / max(1, st["frame_launches"])
        roof["frame_share_of_cell_updates"] = st["frame_cell_updates"] / max(
            1, st["interior_cell_updates"] + st["frame_cell_updates"])

    # ---- the stated error: this (FP32) job against an FP64 run of the same job
    err = None
    if args.precision == "single":
        out32 = job.finish()
        j64 = Job(dict(sim, precision="double"), ctx)
        j64.advance(nsteps)
        out64 = j64.finish()
        j64.close()
        inc = out64["flux"][1][None, :]   # incident flux per wavelength (line after the source)
        line, tr = _line_errors(out32, out64, inc)
        err = {"transmission_abs_max": tr, "dft_line_rel_max": line,
               "against": "FP64 run of the same job on the GPU (the FP64 form is held to the FP64 oracle at "
                          "1e-10 fields / 1e-9 transmission on this grid by tests/test_baseline_parity_gpu.py)",
               "transmission": "T = flux / incident flux (x line after the source), every monitor and wavelength"}

    # ---- end to end through the public API (host arrays in, host arrays out)
    e2e = None
    if not args.no_e2e:
        ectx = Context(local, stream=stream.cuda_stream)
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            fdtd2D(sim, ctx=ectx)   # warm
            ectx.reset_stats()
            _barrier(dist)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                fdtd2D(sim, ctx=ectx)
            torch.cuda.synchronize()
            te = time.perf_counter() - t0
        es = ectx.stats()
        te = _max_over_ranks(dist, te)
        e2e = {"value": cells * nsteps * args.steps * world / te / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": es["h2d_bytes"] // args.steps, "d2h_bytes_per_step": es["d2h_bytes"] // args.steps,
               "ms_per_step": 1e3 * te / args.steps,
               "host_phase_ms": {k: es[k + "_ms"] / args.steps for k in ("setup", "loop", "finish")},
               "note": "orf.fdtd2D(sim): host eps arrays -> material index + tables -> device, "
                       "time loop, DFT lines + fluxes back to host"}
        ectx.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not coupler:
        cpu, dt = cpu_sample(sim, args.cpu_sample_steps)
        cpu["sample"] += f", {dt:.1f} s"
    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.precision == "single" else "f64",
            "data": data,
            "config": {"workload": wl,
                       "cells": cells, "time_steps_per_job": nsteps,
                       "precision": "FP32 fields, FP32+Kahan DFT, FP64 phases" if args.precision == "single"
                       else "FP64", "parallelism": f"replicas x{world}",
                       "l2": l2,
                       "timed_path": "CUDA-graph chunk replays, timing events off"},
            "gpu_launches": launches_per_job * args.steps,
            "roofline": roof, "error_vs_fp64": err, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk.summary(),
            "kernel_ms_one_job": {"interior": st["interior_ms"], "frame": st["frame_ms"],
                                  "flush_check": st["flush_ms"]},
        }
        if coupler:
            line["error_vs_fp64"] = {"note": "this is the FP64 form; tests/test_baseline_parity_gpu.py holds it to "
                                             "the FP64 oracle at 1e-10 fields / 1e-9 transmission on this job"}
    job.close()
    ctx.close()
    return line


def bench_pillar3d(args, rank, world, local, dist):
    """3D TiO2 pillar lattice, 600 x 600 x 300 at 20 nm, 3 DFT planes."""
    import torch
    from opticrcwafdtd_b200 import Context, Job, workloads
    nsteps = args.time_steps or 6000
    nx3, ny3, nz3 = (int(v) for v in args.size3d.split(","))
    sim = workloads.pillar_lattice_sim(nx=nx3, ny=ny3, nz=nz3, steps=nsteps, precision=args.precision,
                                       device=True)   # permittivity by the GPU generator (orf_eps3d)
    cells = sim["x"].size * sim["y"].size * sim["z"].size
    stream = torch.cuda.current_stream()
    ctx = Context(local, stream=stream.cuda_stream)
    job = Job(sim, ctx, dims=3)

    def one_job():
        job.reset()
        job.advance(nsteps)

    for _ in range(args.warmup):
        one_job()
    _barrier(dist)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            one_job()
        ev1.record(stream)
        torch.cuda.synchronize()
    _barrier(dist)
    ms = _max_over_ranks(dist, ev0.elapsed_time(ev1))
    ctx.reset_stats()
    ctx.set_timing(True)
    job.reset()
    job.advance(min(nsteps, 1000))
    torch.cuda.synchronize()
    st = ctx.stats()
    ctx.set_timing(False)
    bpc = BYTES_3D[args.precision]
    roof = _roofline(st, bpc, "k_step3d interior tiles (fused H+E time step, TMA plane ring)")
    if roof:
        if args.precision == "single":
            tpc = ncu_traffic_per_cell_update("step3d_kernel_pillar_lattice.json")
            roof["traffic"] = tpc * roof["cell_updates_per_launch"] if tpc else None
            roof["traffic_note"] = "interior-launch DRAM bytes per cell update from a 300x300x150 capture, scaled"
        cpml = _roofline(st, bpc, "k_step3d CPML tiles", kind="frame")
        roof["cpml_launch_frac"] = cpml["frac"] if cpml else None
        roof["share_of_step_kernels"] = st["interior_ms"] / max(1e-9, st["interior_ms"] + st["frame_ms"])
    clocks = clk.summary()
    value = cells * nsteps * args.steps * world / (ms / 1e3) / 1e6
    # end to end: one fdtd3D(sim) call from the host arrays to host results
    # (set-up: validation, material index, uploads; the time loop; results),
    # after the resident job is released (its device block is reused)
    from opticrcwafdtd_b200 import fdtd3D
    job.close()
    ectx = Context(local)
    ectx.reset_stats()
    t0 = time.perf_counter()
    fdtd3D(sim, ctx=ectx)
    te = time.perf_counter() - t0
    es = ectx.stats()
    e2e = {"value": cells * nsteps / te / 1e6, "unit": UNIT, "ms_per_step": 1e3 * te,
           "h2d_bytes_per_step": es["h2d_bytes"], "d2h_bytes_per_step": es["d2h_bytes"],
           "host_phase_ms": {k: es[k + "_ms"] for k in ("setup", "loop", "finish")}}
    ectx.close()
    line = None
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "e2e": e2e,
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32" if args.precision == "single" else "f64",
                "data": "synthetic (seeded TiO2 pillar radii U[60,180] nm)",
                "config": {"workload": f"3D pillar lattice {nx3}x{ny3}x{nz3} dx=20nm, periodic x/y, 20-cell CPML z, "
                                       f"532 nm plane wave, 3 DFT planes, {nsteps} time steps per job"
                                       + (" (of the workload's 6000)" if nsteps != 6000 else ""),
                           "cells": cells, "time_steps_per_job": nsteps, "parallelism": f"replicas x{world}",
                           "l2": "inputs larger than L2"},
                "roofline": roof, "whole_step_roofline": _whole_frac(value * 1e6, bpc), "clocks": clocks,
                "time_x_median_sm_mhz": (ms / args.steps) * clocks["sm_mhz"] if clocks else None,
                "hbm_gbs_algorithmic": bpc * cells * nsteps * args.steps / (ms / 1e3) / 1e9}
    job.close()
    ctx.close()
    return line


def bench_pillar3d_slabs(args, rank, world, local, dist):
    """The 3D pillar lattice computed as z slabs on one GPU (slab3d.SlabRun:
    one slab job per slab, ghost planes swapped by device copies after every
    step), timed beside the same run on one grid; the DFT planes of both
    compared bit for bit."""
    import numpy as np
    import torch
    from opticrcwafdtd_b200 import Context, Job, SlabRun, workloads
    nsteps = args.time_steps or 300
    nx3, ny3, nz3 = (int(v) for v in args.size3d.split(","))
    sim = workloads.pillar_lattice_sim(nx=nx3, ny=ny3, nz=nz3, steps=nsteps, precision=args.precision, device=True)
    cells = nx3 * ny3 * nz3
    run = SlabRun(sim, args.slabs, local)
    stream = torch.cuda.current_stream()
    ctx = Context(local, stream=stream.cuda_stream)
    job = Job(sim, ctx, dims=3)

    def timed(fn, sync_stream):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(sync_stream)
        for _ in range(args.steps):
            fn()
        ev1.record(sync_stream)
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1)

    def slab_run():
        run.reset()
        run.run()

    def one_grid():
        job.reset()
        job.advance(nsteps)

    with ClockSampler(local) as clk:
        ms_slab = timed(slab_run, run.stream)
        ms_one = timed(one_grid, stream)
    out_s = run.finish()
    out_1 = job.finish()
    same = all(np.array_equal(a[k], b[k]) for a, b in zip(out_s["mon"], out_1["mon"]) for k in ("Ea", "Eb", "Ha", "Hb"))
    v_slab = cells * nsteps * args.steps / (ms_slab / 1e3) / 1e6
    v_one = cells * nsteps * args.steps / (ms_one / 1e3) / 1e6
    bpc = BYTES_3D[args.precision]
    line = {"metric": METRIC, "value": v_slab, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_slab / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "single" else "f64",
            "data": "synthetic (seeded TiO2 pillar radii U[60,180] nm)",
            "config": {"workload": f"3D pillar lattice {nx3}x{ny3}x{nz3} as {args.slabs} z slabs on one GPU "
                                   f"(ghost planes swapped after every step), {nsteps} time steps",
                       "cells": cells, "slabs": [[q.z0, q.z1] for q in run.slabs], "parallelism": "z slabs x1 GPU",
                       "l2": "inputs larger than L2"},
            "whole_step_roofline": _whole_frac(v_slab * 1e6, bpc),
            "one_grid_value": v_one, "slab_over_one_grid": v_slab / v_one,
            "monitors_bitwise_equal_one_grid": bool(same),
            # per inner cut: Ex Ey Ez planes up, Ex Ey planes down (pitch x ny each)
            "swap_bytes_per_step": 5 * ((nx3 + 31) // 32 * 32) * ny3 * (4 if args.precision == "single" else 8)
                                   * (len(run.slabs) - 1),
            "clocks": clk.summary()}
    run.close()
    job.close()
    ctx.close()
    return line


def bench_coupler_batch(args, rank, world, local, dist):
    """256 uneven 2D TE grating couplers advanced together (orf_batch2d_run)."""
    import numpy as np
    import torch
    from opticrcwafdtd_b200 import Context, fdtd2D_batch, workloads
    nsteps = args.time_steps or 10000
    sims = workloads.coupler_batch_sims(n=args.batch, steps=nsteps, precision=args.precision)
    cu = sum(s["x"].size * s["z"].size for s in sims) * nsteps
    stream = torch.cuda.current_stream()
    ctx = Context(local, stream=stream.cuda_stream)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        for w in range(args.warmup):
            # the first warm-up call autotunes (variant, fused depth) on a batched sample of instances
            fdtd2D_batch(sims, ctx, autotune=(w == 0))
        _barrier(dist)
        torch.cuda.synchronize()
        with ClockSampler(local) as clk:
            t0 = time.perf_counter()
            for _ in range(args.steps):
                outs = fdtd2D_batch(sims, ctx)
            torch.cuda.synchronize()
            te = time.perf_counter() - t0
        _barrier(dist)
        te = _max_over_ranks(dist, te)
        # per-launch events on one more call: the step kernels' split and roofline
        ctx.reset_stats()
        ctx.set_timing(True)
        fdtd2D_batch(sims, ctx)
        torch.cuda.synchronize()
        st = ctx.stats()
        ctx.set_timing(False)
        # coupling-efficiency error of 8 seeded instances against their FP64 runs
        pick = sorted(set(int(round(v)) for v in np.linspace(0, len(sims) - 1, 8)))
        eta_err = None
        if args.precision == "single":
            o64 = fdtd2D_batch([dict(sims[q], precision="double") for q in pick], ctx)
            errs = [float(np.max(np.abs(workloads.coupler_instance_eta(outs[q], sims[q]) -
                                        workloads.coupler_instance_eta(o, sims[q])))) for q, o in zip(pick, o64)]
            eta_err = {"jobs": len(errs), "max": max(errs),
                       "against": "FP64 batched run of the same instances on the GPU (held to the FP64 oracle by "
                                  "tests/test_baseline_parity_gpu.py)",
                       "eta": "fiber coupling efficiency, theta 5..15 deg, fiber centre every 0.5 um, every lambda"}
    value = cu * args.steps * world / te / 1e6
    bpc = 25 if args.precision == "single" else 49
    roof = _roofline(st, bpc, "k_step2d_fast (CPML frame tiles, PML=true)", kind="frame")
    inter = _roofline(st, bpc, "k_step2d_fast (interior tiles)")
    step_ms = st["interior_ms"] + st["frame_ms"]
    if roof:
        roof["interior_launch_frac"] = inter["frac"] if inter else None
        roof["frame_share_of_step_time"] = st["frame_ms"] / max(1e-9, step_ms)
        roof["frame_share_of_cell_updates"] = st["frame_cell_updates"] / max(
            1, st["interior_cell_updates"] + st["frame_cell_updates"])
        roof["step_kernels_frac"] = (bpc * (st["interior_cell_updates"] + st["frame_cell_updates"]) /
                                     (step_ms / 1e3) / 1e9) / roof["peak"]
    line = None
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": te * 1e3 / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32" if args.precision == "single" else "f64",
                "data": "synthetic (seeded grating parameters)",
                "config": {"workload": f"{args.batch} 2D TE grating couplers 600-1200 x 250-350 dx=20nm, "
                                       f"51-lambda DFT, {nsteps} steps each, one orf_batch2d_run per step",
                           "tuning": "orf_autotune2d on a batched sample of 32 instances during warm-up",
                           "jobs_per_s": args.batch * args.steps * world / te, "parallelism": f"replicas x{world}",
                           "timed_path": "host sims -> device -> results on host (end to end)"},
                "jobs_per_s": args.batch * args.steps * world / te,
                "roofline": roof, "whole_job_roofline": _whole_frac(value * 1e6, bpc),
                "eta_err_vs_fp64": eta_err, "clocks": clk.summary(), "tuning_choice": getattr(ctx, "tuned", None),
                "host_phase_ms": {"setup": st["setup_ms"], "loop": st["loop_ms"], "finish": st["finish_ms"]}}
    ctx.close()
    return line


def _serve_run(srv, jobs, t_arrive):
    """Submit jobs at their arrival times (seconds after the start) and step
    the server until all are done; returns (tickets, makespan)."""
    tickets = []
    nxt = 0
    t0 = srv.clock()
    while True:
        now = srv.clock() - t0
        while nxt < len(jobs) and t_arrive[nxt] <= now:
            tickets.append(srv.submit(jobs[nxt]["sim"], dims=jobs[nxt]["dims"]))
            nxt += 1
        q, r = srv.pending()
        if q == 0 and r == 0:
            if nxt >= len(jobs):
                break
            time.sleep(max(0.0, min(0.05, t_arrive[nxt] - now)))
            continue
        srv.step()
    return tickets, srv.clock() - t0


def bench_serve(args, rank, world, local, dist):
    """Poisson stream of mixed 2D / 3D jobs through the serving loop, at a
    stated fraction of the capacity measured on a saturated sample of the same
    job distribution."""
    import numpy as np
    import torch
    from opticrcwafdtd_b200 import Context, Server, fdtd2D_batch, fdtd3D, workloads
    warnings.simplefilter("ignore")
    cells = (2e5, args.serve_max_cells)
    ctx = Context(local, stream=torch.cuda.current_stream().cuda_stream)
    phase = {}
    t = time.perf_counter()
    # 3D permittivities from the GPU generator (bitwise the host generator's)
    stream_jobs = workloads.serve_stream(n_jobs=args.serve_jobs, rate=1.0, seed=5 + rank, cells=cells, device=ctx)
    cap_jobs = workloads.serve_stream(n_jobs=args.serve_capacity_jobs, rate=1.0, seed=1000 + rank, cells=cells,
                                      device=ctx)
    phase["build_sims"] = time.perf_counter() - t
    cu = [j["cells"] * j["steps"] for j in stream_jobs]
    # warm the kernels once on a small job of each kind
    warm = workloads.serve_stream(n_jobs=4, seed=99, cells=(2e5, 4e5), steps=(200, 300), frac3d=0.5)
    srv = Server(ctx, macro_steps=args.serve_macro)
    for j in warm:
        srv.submit(j["sim"], dims=j["dims"])
    srv.drain()
    srv.close()
    # capacity: a sample of the same distribution submitted all at once
    t = time.perf_counter()
    srv = Server(ctx, macro_steps=args.serve_macro)
    _, cap_span = _serve_run(srv, cap_jobs, [0.0] * len(cap_jobs))
    srv.close()
    phase["capacity"] = time.perf_counter() - t
    cap_cu_s = sum(j["cells"] * j["steps"] for j in cap_jobs) / cap_span
    capacity = cap_cu_s / (sum(cu) / len(cu))   # jobs/s of this stream's mean job
    rate = args.serve_rate if args.serve_rate > 0 else args.serve_load * capacity
    # the stream: the seeded exponential gaps of serve_stream, scaled to the rate
    t_arr = [j["t"] / rate for j in stream_jobs]
    srv = Server(ctx, macro_steps=args.serve_macro)
    _barrier(dist)
    torch.cuda.synchronize()
    t = time.perf_counter()
    with ClockSampler(local) as clk:
        tickets, span = _serve_run(srv, stream_jobs, t_arr)
    phase["stream"] = time.perf_counter() - t
    t = time.perf_counter()
    infos = [srv.info(t) for t in tickets]
    lat = np.array([i["t_done"] - i["t_submit"] for i in infos])
    bytes_alg = sum(c * (BYTES_3D["single"] if j["dims"] == 3 else 25) for c, j in zip(cu, stream_jobs))
    peak, peak_kind = measured_peaks()
    # per-job error against the FP64 plain form: coupling efficiency of a
    # seeded sample of the 2D couplers (every k-th), flux transmission of the
    # two smallest 3D jobs
    idx2 = [q for q, j in enumerate(stream_jobs) if j["dims"] == 2]
    idx3 = sorted((q for q, j in enumerate(stream_jobs) if j["dims"] == 3), key=lambda q: cu[q])[:2]
    k = max(1, int(round(1.0 / max(1e-9, args.serve_check_frac))))
    chk2 = idx2[::k]
    eta_errs = []
    if chk2:
        o64 = fdtd2D_batch([dict(stream_jobs[q]["sim"], precision="double") for q in chk2], ctx)
        for q, o in zip(chk2, o64):
            o32 = srv.result(tickets[q])
            s = stream_jobs[q]["sim"]
            eta_errs.append(float(np.max(np.abs(workloads.coupler_instance_eta(o32, s) -
                                                workloads.coupler_instance_eta(o, s)))))
    t_errs = []
    for q in idx3:
        o32 = srv.result(tickets[q])
        o64 = fdtd3D(dict(stream_jobs[q]["sim"], precision="double"), ctx)
        f32, f64 = np.asarray(o32["flux"]), np.asarray(o64["flux"])
        t_errs.append(float(np.max(np.abs(f32 - f64)) / max(1e-300, np.max(np.abs(f64)))))
    srv.close()
    ctx.close()
    phase["fp64_checks"] = time.perf_counter() - t
    if rank != 0:
        return None
    n2 = len(idx2)
    return {"metric": "jobs/s", "value": len(tickets) * world / span, "unit": "jobs/s", "n_gpus": world,
            "steps": 1, "warmup": 1, "ms_per_step": span * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded Poisson stream, random grating / pillar geometries)",
            "config": {"workload": f"served stream of {len(tickets)} jobs ({n2} 2D grating couplers, "
                                   f"{len(tickets) - n2} 3D pillar lattices), Poisson arrivals at "
                                   f"{rate:.3f} jobs/s = {rate / capacity:.2f} x the measured capacity, cells "
                                   f"log-uniform [2e5, {args.serve_max_cells:.0e}], steps U[2000, 20000], FP32",
                       "macro_steps": args.serve_macro, "parallelism": f"replicas x{world}",
                       "capacity_sample": f"{len(cap_jobs)} jobs of the same distribution submitted at once"},
            "capacity_jobs_per_s": capacity, "capacity_mcell_updates_per_s": cap_cu_s / 1e6, "rate": rate,
            "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                          "max": float(lat.max())},
            "mcell_updates_per_s": sum(cu) / span / 1e6, "makespan_s": span,
            "roofline": {"bound": "hbm", "achieved": bytes_alg / span / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": bytes_alg / span / 1e9 / peak, "peak_source": peak_kind,
                         "note": "algorithmic bytes of all jobs (2D TE FP32 25 B, 3D FP32 51 B per cell update) over "
                                 "the makespan, under the stated load"},
            "eta_err_vs_fp64": {"jobs": len(eta_errs), "of_2d_jobs": n2, "max": max(eta_errs) if eta_errs else None,
                                "sample": f"every {k}-th 2D coupler job, FP64 batched run on the GPU"},
            "flux_T_err_vs_fp64_3d": {"jobs": len(t_errs), "max": max(t_errs) if t_errs else None,
                                      "sample": "the two smallest 3D jobs, T = flux / largest |flux|"},
            "phase_s": phase, "clocks": clk.summary()}


def bench_fdfd(args, rank, world, local, dist):
    """The 2D TE frequency-domain solver (orf.fdfd2D, toolbox/+orf/fdfd2D.m)
    on the reference's straight-guide problem: SOI slab, 501 x 221 points at
    20 nm, 30-cell PML, TE0 source; one factorisation, one solve, one adjoint
    solve, against the FDFD oracle (scipy sparse LU, one host thread)."""
    import numpy as np
    import torch
    import opticrcwafdtd_b200 as orf
    from opticrcwafdtd_b200 import workloads
    x, z, epsr, lam, J, m, win = workloads.fdfd_straight_guide()
    ctx = orf.Context(local)
    g = np.conj(J)
    for _ in range(max(1, args.warmup)):
        orf.fdfd2D(x, z, epsr, lam, J, ctx=ctx).close()
    reps = max(1, args.steps)
    tf = ts = ta = 0.0
    with ClockSampler(local) as clk:
        for _ in range(reps):
            t0 = time.perf_counter()
            o = orf.fdfd2D(x, z, epsr, lam, J, ctx=ctx)   # factorisation + the first solve
            t1 = time.perf_counter()
            o.solve(J)
            t2 = time.perf_counter()
            lam_ = o.adjoint(g)
            t3 = time.perf_counter()
            tf += (t1 - t0) - (t2 - t1)
            ts += t2 - t1
            ta += t3 - t2
            E = o.E
            info = o.info()
            o.close()
    torch.cuda.synchronize()
    tf, ts, ta = 1e3 * tf / reps, 1e3 * ts / reps, 1e3 * ta / reps
    mb, nb = info["block"], info["blocks"]
    sweep_bytes = 2 * nb * mb * mb * 16          # the two sweeps read every block inverse once
    peak, src = measured_peaks()
    line = {"metric": "fdfd2D factor + solve", "value": tf + ts, "unit": "ms", "n_gpus": 1, "steps": reps,
            "warmup": max(1, args.warmup), "ms_per_step": tf + ts + ta, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic (SOI slab, TE0 mode source)",
            "config": {"workload": "FDFD 2D TE SOI slab 501x221 dx=20nm, 30-cell PML, one factorisation, "
                                   "one solve, one adjoint solve", "block": mb, "blocks": nb,
                       "cluster_ctas": info["cluster"]},
            "factor_ms": tf, "solve_ms": ts, "adjoint_ms": ta,
            "factor_gflops": 8.0 * nb * mb ** 3 / (tf / 1e3) / 1e9,
            "solve_roofline": {"bound": "hbm", "achieved": sweep_bytes / (ts / 1e3) / 1e9, "peak": peak,
                               "unit": "GB/s", "frac": sweep_bytes / (ts / 1e3) / 1e9 / peak, "peak_source": src,
                               "note": "block inverses read by the two sweeps; host copies of J and E included"},
            "clocks": clk.summary()}
    if not args.no_cpu_baseline:
        from oracle.fdfd import fdfd2D as ofdfd
        t0 = time.perf_counter()
        r = ofdfd(x, z, epsr, lam, J)
        t1 = time.perf_counter()
        ra = r.adjoint(g)
        t2 = time.perf_counter()
        rel = lambda a, b: float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))
        line["cpu_baseline"] = {"value": 1e3 * (t1 - t0), "unit": "ms", "cores": 1, "kind": "port",
                                "sample": "the same factorisation + solve (scipy sparse LU, SuperLU)",
                                "adjoint_ms": 1e3 * (t2 - t1)}
        line["error_vs_oracle"] = {"E_rel_l2": rel(E, r.E), "adjoint_rel_l2": rel(lam_, ra)}
    ctx.close()
    return line


WORKLOADS = {"pixel2d": bench_pixel2d, "coupler": bench_pixel2d, "pillar3d": bench_pillar3d,
             "pillar3d_slabs": bench_pillar3d_slabs,
             "coupler_batch": bench_coupler_batch, "serve": bench_serve, "fdfd": bench_fdfd}


def run_forms(args, local):
    """The sub-records of the headline line (N = 1): every other form of the
    engine, each at its workload's shape with its own timing and clocks."""
    subs = [
        ("c1_coupler_fp64", "coupler", dict(time_steps=8000, steps=20, warmup=3, precision="double",
                                            no_cpu_baseline=True)),
        ("c3_pillar_fp32", "pillar3d", dict(time_steps=1000, steps=3, warmup=3, precision="single",
                                            size3d="600,600,300")),
        ("c3_pillar_fp64", "pillar3d", dict(time_steps=1000, steps=3, warmup=3, precision="double",
                                            size3d="600,600,300")),
        ("c3_pillar_fp32_2slabs", "pillar3d_slabs", dict(time_steps=300, steps=3, warmup=3, precision="single",
                                                        size3d="600,600,300", slabs=2)),
        ("c4_coupler_batch", "coupler_batch", dict(time_steps=10000, steps=3, warmup=3, precision="single",
                                                   batch=256)),
        ("c5_served", "serve", dict()),
        ("fdfd2d", "fdfd", dict(steps=3, warmup=1)),
    ]
    out = {}
    for key, wl, kw in subs:
        a = argparse.Namespace(**vars(args))
        a.workload = wl
        a.__dict__.update(kw)
        t = time.perf_counter()
        try:
            rec = WORKLOADS[wl](a, 0, 1, local, None)
        except Exception as e:  # noqa: BLE001 - a failed sub-record must not hide the headline
            rec = {"error": f"{type(e).__name__}: {e}"}
        rec["wall_s"] = time.perf_counter() - t
        out[key] = rec
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    rank, world, local = dist_env()
    dist = _init_dist(local, world)
    line = WORKLOADS[args.workload](args, rank, world, local, dist)
    if rank == 0 and line is not None and world == 1 and args.workload == "pixel2d" and not args.no_forms:
        line.update(run_forms(args, local))
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
