#!/usr/bin/env python
"""Benchmark of the B200 Yee-FDTD engine on the 2D TM 4000 x 1500 pixel-region workload.

Workload (one bench "step" = one whole FDTD job): 2D TM, 4000 x 1500 cells at
dx = 10 nm with 20-cell CPML, a seeded Bernoulli Si/SiO2 pixel design region
in an SOI waveguide, TM0 mode source, 101-wavelength DFT monitors over
1.5-1.6 um, 30000 time steps, FP32 fields with Kahan-compensated FP32 DFT
sums.  The fields (2 x 72 MB ping-pong + 12 MB material index) exceed the
126 MB L2, so no flush is needed between timed steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload pixel2d|pillar3d|coupler_batch|serve]

pixel2d (the default) is the headline above.  The other workloads measure
the remaining paths, each printing its own JSON line: pillar3d (3D TiO2
pillar lattice, 600 x 600 x 300, 6000 steps), coupler_batch (256 uneven 2D
grating couplers, 10000 steps each, one batched call per step) and serve (a
Poisson stream of mixed 2D / 3D jobs through the serving loop: jobs/s, p50 /
p99 latency, flux error of sampled jobs against the FP64 form).

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

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "Yee Mcells/s"
UNIT = "Mcell-updates/s"
BYTES_PER_CELL_UPDATE = {("TM", "single"): 26, ("TM", "double"): 50, ("TE", "single"): 25, ("TE", "double"): 49}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="single", choices=["single", "double"])
    ap.add_argument("--time-steps", type=int, default=30000, help="FDTD time steps per job (the workload: 30000)")
    ap.add_argument("--cpu-sample-steps", type=int, default=300)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", default="pixel2d", choices=["pixel2d", "coupler", "pillar3d", "coupler_batch", "serve"],
                    help="pixel2d is the headline; the others measure the 3D, batched and served paths")
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--size3d", default="600,600,300", help="pillar3d grid NX,NY,NZ (smaller for profiling)")
    ap.add_argument("--serve-jobs", type=int, default=32)
    ap.add_argument("--serve-rate", type=float, default=0.33)
    ap.add_argument("--serve-max-cells", type=float, default=5e7)
    ap.add_argument("--serve-macro", type=int, default=500)
    ap.add_argument("--serve-check", type=int, default=4)
    return ap.parse_args()


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
        self.path = os.path.join(tempfile.gettempdir(), f"orf_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
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


def cpu_baseline(sim, sample_steps):
    """The oracle (C++ restatement, FP32 fields as the GPU form) on all host cores."""
    import oracle
    s = dict(sim)
    S = 0.99 / math.sqrt(2) * 0.01
    s["maxTime"] = sample_steps * S
    threads = os.cpu_count() or 1
    t = time.perf_counter()
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        oracle.fdtd2D(s, threads=threads)
    dt = time.perf_counter() - t
    cells = s["epsX"].shape[0] * (s["epsZ"].shape[1])
    return {"value": cells * sample_steps / dt / 1e6, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"TM pixel-region grid {cells} cells, {sample_steps} of 30000 time steps, "
                      f"{s['precision']} fields, {dt:.1f} s"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from opticrcwafdtd_b200 import workloads
    sim = workloads.pixel_region_sim(precision=args.precision)
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(sim, max(20, args.cpu_sample_steps // 2))
        if i >= args.warmup:
            vals.append(r["value"])
    v = statistics.mean(vals)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "dtype": "f32" if args.precision == "single" else "f64",
        "data": "synthetic (seeded Bernoulli Si/SiO2 pixel map, 4000x1500)",
        "config": {"workload": "2D TM pixel region 4000x1500 dx=10nm, 101-lambda DFT, 30000 steps (bounded sample)"},
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
    """Roofline of the dominant step kernel from its per-launch CUDA events."""
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


def bench_pixel2d(args, rank, world, local, dist):
    """Headline: whole 2D TM pixel-region jobs, device-resident inputs
    (--workload coupler: the 800 x 300 FP64 TE grating coupler instead)."""
    import torch
    from opticrcwafdtd_b200 import Context, Job, fdtd2D, workloads

    coupler = args.workload == "coupler"
    if coupler:
        if args.time_steps == 30000:
            args.time_steps = 8000
        args.precision = "double"
        sim = workloads.coupler_sim(precision="double", steps=args.time_steps)
        pol, nx, nz = "TE", sim["eps"].shape[0], sim["eps"].shape[1]
        data = "synthetic (SOI grating coupler: 20 x 630 nm periods, ff 0.5, 70 nm etch)"
        wl = ("2D TE SOI grating coupler 800x300 dx=20nm 20-cell CPML, TE0 source, 51-lambda DFT, "
              f"{args.time_steps} time steps per job, FP64")
        l2 = "working set below L2 (this small case runs from L2)"
    else:
        sim = workloads.pixel_region_sim(precision=args.precision, steps=args.time_steps)
        pol, nx, nz = "TM", sim["epsX"].shape[0], sim["epsZ"].shape[1]
        data = "synthetic (seeded Bernoulli Si/SiO2 pixel map, 4000x1500)"
        wl = ("2D TM pixel region 4000x1500 dx=10nm 20-cell CPML, TM0 source, "
              "101-lambda DFT (3 x-lines, 2 z-lines), 30000 time steps per job")
        l2 = "inputs larger than L2 (156 MB working set > 126 MB)"
    cells = nx * nz
    stream = torch.cuda.current_stream()
    ctx = Context(local, stream=stream.cuda_stream)
    job = Job(sim, ctx)
    nsteps = args.time_steps

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
    launches_per_job = None

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
    if roof and not coupler:
        tpc = ncu_traffic_per_cell_update()
        roof["traffic"] = tpc * roof["cell_updates_per_launch"] if tpc else None
        roof["share_of_step_kernels"] = st["interior_ms"] / max(1e-9, st["interior_ms"] + st["frame_ms"])
        roof["frame_kernel_avg_launch_ms"] = st["frame_ms"] / max(1, st["frame_launches"])

    # ---- end to end through the public API (host arrays in, host arrays out)
    e2e = None
    if not args.no_e2e:
        ectx = Context(local, stream=stream.cuda_stream)
        import warnings
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
               "note": "orf.fdtd2D(sim): host eps arrays -> material index + tables -> device, "
                       "time loop, DFT lines + fluxes back to host"}
        ectx.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not coupler:
        cpu = cpu_baseline(sim, args.cpu_sample_steps)
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
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk.summary(),
            "kernel_ms_one_job": {"interior": st["interior_ms"], "frame": st["frame_ms"],
                                  "flush_check": st["flush_ms"]},
        }
    job.close()
    ctx.close()
    return line


def bench_pillar3d(args, rank, world, local, dist):
    """3D TiO2 pillar lattice, 600 x 600 x 300 at 20 nm, 3 DFT planes."""
    import torch
    from opticrcwafdtd_b200 import Context, Job, workloads
    nsteps = args.time_steps if args.time_steps != 30000 else 6000
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
    bpc = 51 if args.precision == "single" else 99
    roof = _roofline(st, bpc, "k_step3d (fused H+E time step, TMA plane ring; interior and CPML tile launches)")
    if roof and args.precision == "single":
        tpc = ncu_traffic_per_cell_update("step3d_kernel_pillar_lattice.json")
        roof["traffic"] = tpc * roof["cell_updates_per_launch"] if tpc else None
        roof["traffic_note"] = "interior-launch DRAM bytes per cell update from a 300x300x150 capture, scaled"
    line = None
    if rank == 0:
        line = {"metric": METRIC, "value": cells * nsteps * args.steps * world / (ms / 1e3) / 1e6, "unit": UNIT,
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32" if args.precision == "single" else "f64",
                "data": "synthetic (seeded TiO2 pillar radii U[60,180] nm)",
                "config": {"workload": f"3D pillar lattice {nx3}x{ny3}x{nz3} dx=20nm, periodic x/y, 20-cell CPML z, "
                                       "532 nm plane wave, 3 DFT planes", "cells": cells,
                           "time_steps_per_job": nsteps, "parallelism": f"replicas x{world}",
                           "l2": "inputs larger than L2"},
                "roofline": roof, "clocks": clk.summary(),
                "hbm_gbs_algorithmic": bpc * cells * nsteps * args.steps / (ms / 1e3) / 1e9}
    job.close()
    ctx.close()
    return line


def bench_coupler_batch(args, rank, world, local, dist):
    """256 uneven 2D TE grating couplers advanced together (orf_batch2d_run)."""
    import torch
    from opticrcwafdtd_b200 import Context, fdtd2D_batch, workloads
    nsteps = args.time_steps if args.time_steps != 30000 else 10000
    sims = workloads.coupler_batch_sims(n=args.batch, steps=nsteps, precision=args.precision)
    cu = sum(s["x"].size * s["z"].size for s in sims) * nsteps
    stream = torch.cuda.current_stream()
    ctx = Context(local, stream=stream.cuda_stream)
    import warnings
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
                fdtd2D_batch(sims, ctx)
            torch.cuda.synchronize()
            te = time.perf_counter() - t0
    _barrier(dist)
    te = _max_over_ranks(dist, te)
    line = None
    if rank == 0:
        line = {"metric": METRIC, "value": cu * args.steps * world / te / 1e6, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": te * 1e3 / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32" if args.precision == "single" else "f64",
                "data": "synthetic (seeded grating parameters)",
                "config": {"workload": f"{args.batch} 2D TE grating couplers 600-1200 x 250-350 dx=20nm, "
                                       f"51-lambda DFT, {nsteps} steps each, one orf_batch2d_run per step",
                           "tuning": "orf_autotune2d on a batched sample of 32 instances during warm-up",
                           "jobs_per_s": args.batch * args.steps * world / te, "parallelism": f"replicas x{world}",
                           "timed_path": "host sims -> device -> results on host (end to end)"},
                "clocks": clk.summary()}
    ctx.close()
    return line


def bench_serve(args, rank, world, local, dist):
    """Poisson stream of mixed 2D / 3D jobs through the serving loop."""
    import numpy as np
    import torch
    from opticrcwafdtd_b200 import Context, Server, fdtd2D, fdtd3D, workloads
    stream_jobs = workloads.serve_stream(n_jobs=args.serve_jobs, rate=args.serve_rate, seed=5 + rank,
                                         cells=(2e5, args.serve_max_cells))
    ctx = Context(local, stream=torch.cuda.current_stream().cuda_stream)
    import warnings
    warnings.simplefilter("ignore")
    # warm the kernels once on a small job of each kind
    warm = workloads.serve_stream(n_jobs=4, seed=99, cells=(2e5, 4e5), steps=(200, 300), frac3d=0.5)
    srv = Server(ctx, macro_steps=args.serve_macro)
    for j in warm:
        srv.submit(j["sim"], dims=j["dims"])
    srv.drain()
    srv.close()
    srv = Server(ctx, macro_steps=args.serve_macro)
    _barrier(dist)
    torch.cuda.synchronize()
    tickets = []
    nxt = 0
    with ClockSampler(local) as clk:
        t0 = srv.clock()
        while True:
            now = srv.clock() - t0
            while nxt < len(stream_jobs) and stream_jobs[nxt]["t"] <= now:
                tickets.append(srv.submit(stream_jobs[nxt]["sim"], dims=stream_jobs[nxt]["dims"]))
                nxt += 1
            q, r = srv.pending()
            if q == 0 and r == 0:
                if nxt >= len(stream_jobs):
                    break
                time.sleep(max(0.0, min(0.05, stream_jobs[nxt]["t"] - now)))
                continue
            srv.step()
        span = srv.clock() - t0
    infos = [srv.info(t) for t in tickets]
    lat = np.array([i["t_done"] - i["t_submit"] for i in infos])
    cu = sum(j["cells"] * j["steps"] for j in stream_jobs)
    # per-job error of the FP32 results against the FP64 plain form, on a sample
    errs = []
    for q in range(min(args.serve_check, len(tickets))):
        j = stream_jobs[q]
        s64 = dict(j["sim"], precision="double")
        o32 = srv.result(tickets[q])
        o64 = fdtd2D(s64, ctx) if j["dims"] == 2 else fdtd3D(s64, ctx)
        f32, f64 = np.asarray(o32["flux"]), np.asarray(o64["flux"])
        errs.append(float(np.max(np.abs(f32 - f64)) / max(1e-300, np.max(np.abs(f64)))))
    srv.close()
    ctx.close()
    if rank != 0:
        return None
    return {"metric": "jobs/s", "value": len(tickets) * world / span, "unit": "jobs/s", "n_gpus": world,
            "steps": 1, "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded Poisson stream, random grating / pillar geometries)",
            "config": {"workload": f"served stream of {len(tickets)} jobs, Poisson rate {args.serve_rate}/s, "
                                   f"80% 2D grating couplers / 20% 3D pillar lattices, cells log-uniform "
                                   f"[2e5, {args.serve_max_cells:.0e}], steps U[2000, 20000], FP32",
                       "macro_steps": args.serve_macro, "parallelism": f"replicas x{world}"},
            "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                          "max": float(lat.max())},
            "mcell_updates_per_s": cu / span / 1e6, "makespan_s": span,
            "flux_rel_err_vs_fp64": {"jobs": len(errs), "max": max(errs) if errs else None},
            "clocks": clk.summary()}


WORKLOADS = {"pixel2d": bench_pixel2d, "coupler": bench_pixel2d, "pillar3d": bench_pillar3d,
             "coupler_batch": bench_coupler_batch, "serve": bench_serve}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    rank, world, local = dist_env()
    dist = _init_dist(local, world)
    line = WORKLOADS[args.workload](args, rank, world, local, dist)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
