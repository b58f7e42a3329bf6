#!/usr/bin/env python
"""Benchmark of the B200 Yee-FDTD engine on the 2D TM 4000 x 1500 pixel-region workload.

Workload (one bench "step" = one whole FDTD job): 2D TM, 4000 x 1500 cells at
dx = 10 nm with 20-cell CPML, a seeded Bernoulli Si/SiO2 pixel design region
in an SOI waveguide, TM0 mode source, 101-wavelength DFT monitors over
1.5-1.6 um, 30000 time steps, FP32 fields with Kahan-compensated FP32 DFT
sums.  The fields (2 x 72 MB ping-pong + 12 MB material index) exceed the
126 MB L2, so no flush is needed between timed steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

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


def ncu_traffic_per_cell_update():
    """DRAM bytes per cell update of the interior kernel from the committed ncu summary."""
    p = os.path.join(HERE, "profiles", "interior_kernel_tm_pixel_4000x1500.json")
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
        self.path = os.path.join(HERE, "gpurun_out", f".clocks_{os.getpid()}.csv")

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


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    rank, world, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    from opticrcwafdtd_b200 import Context, Job, fdtd2D, workloads

    sim = workloads.pixel_region_sim(precision=args.precision, steps=args.time_steps)
    nx, nz = sim["epsX"].shape[0], sim["epsZ"].shape[1]
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
    ctx.reset_stats()
    ctx.set_timing(True)

    def barrier():
        if dist is not None:
            dist.barrier()

    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            one_job()
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    st = ctx.stats()
    ctx.set_timing(False)
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = cells * nsteps * args.steps * world / (ms / 1e3) / 1e6
    launches = st["interior_launches"] + st["frame_launches"] + st["flush_launches"]

    # ---- roofline of the dominant (interior) kernel
    peak, peak_kind = measured_peaks()
    bpc = BYTES_PER_CELL_UPDATE[("TM", args.precision)]
    roof = None
    if st["interior_ms"] > 0:
        per_launch_bytes = bpc * st["interior_cell_updates"] / st["interior_launches"]
        launch_s = st["interior_ms"] / 1e3 / st["interior_launches"]
        achieved = per_launch_bytes / launch_s / 1e9
        tpc = ncu_traffic_per_cell_update()
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
                "traffic": (tpc * st["interior_cell_updates"] / st["interior_launches"]) if tpc else None,
                "kernel": "k_step2d_fast (interior tiles)",
                "algorithmic_bytes_per_cell_update": bpc,
                "avg_launch_ms": launch_s * 1e3,
                "share_of_step_kernels": st["interior_ms"] / max(1e-9, st["interior_ms"] + st["frame_ms"]),
                "frame_kernel_avg_launch_ms": st["frame_ms"] / max(1, st["frame_launches"])}

    # ---- end to end through the public API (host arrays in, host arrays out)
    e2e = None
    if not args.no_e2e:
        ectx = Context(local, stream=stream.cuda_stream)
        import warnings
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            fdtd2D(sim, ctx=ectx)   # warm
            ectx.reset_stats()
            barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                out = fdtd2D(sim, ctx=ectx)
            torch.cuda.synchronize()
            te = time.perf_counter() - t0
        es = ectx.stats()
        if dist is not None:
            t = torch.tensor([te], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            te = float(t.item())
        e2e = {"value": cells * nsteps * args.steps * world / te / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": es["h2d_bytes"] // args.steps, "d2h_bytes_per_step": es["d2h_bytes"] // args.steps,
               "note": "orf.fdtd2D(sim): host eps arrays -> material index + tables -> device, "
                       "time loop, DFT lines + fluxes back to host"}
        ectx.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(sim, args.cpu_sample_steps)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.precision == "single" else "f64",
            "data": "synthetic (seeded Bernoulli Si/SiO2 pixel map, 4000x1500)",
            "config": {"workload": "2D TM pixel region 4000x1500 dx=10nm 20-cell CPML, TM0 source, "
                                   "101-lambda DFT (3 x-lines, 2 z-lines), 30000 time steps per job",
                       "cells": cells, "time_steps_per_job": nsteps,
                       "precision": "FP32 fields, FP32+Kahan DFT, FP64 phases" if args.precision == "single"
                       else "FP64", "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (156 MB working set > 126 MB)"},
            "gpu_launches": launches,
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk.summary(),
            "kernel_ms": {"interior": st["interior_ms"], "frame": st["frame_ms"], "flush_check": st["flush_ms"]},
        }
        print(json.dumps(line), flush=True)
    job.close()
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
