"""Runs small 2D sims through the checked build of the library (selected by
ORF_FDTD_LIB in the environment; see tests/test_check_build_gpu.py) and
prints one JSON line: the out-of-bounds accesses the build counted, and the
largest error against the oracle.  Test infrastructure only."""
import ctypes as C
import json
import os
import sys
import warnings

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from opticrcwafdtd_b200 import Context, Job, _lib, fdtd2D_batch, workloads  # noqa: E402
from tests import cases  # noqa: E402


def _rel(a, b):
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (n if n > 0 else 1.0))


def main():
    warnings.simplefilter("ignore")
    lib = _lib.load()
    assert os.path.basename(_lib.LIB_PATH) == "liborf_fdtd_check.so", _lib.LIB_PATH
    cnt = C.c_uint64()
    _lib.check(lib.orf_check_violations(C.byref(cnt), 1), "check counter")
    worst64, worst32, runs = 0.0, 0.0, 0
    for pol, per in (("TE", False), ("TM", False), ("TE", True), ("TM", True)):
        for prec in ("double", "single"):
            sim = cases.mixed_te_sim(nx=300, nz=170, steps=160, seed=7, pol=pol, periodic=per, precision=prec)
            ref = oracle.fdtd2D(dict(sim, precision="double"), fields=True)
            for tsteps, variant in ((0, 0), (3, 1), (8, 2), (10, 1)):
                ctx = Context(0)
                ctx.set_tuning(tsteps=tsteps, variant=variant)
                job = Job(sim, ctx)
                job.advance(10 ** 9)
                f = job.fields()
                job.finish()
                job.close()
                ctx.close()
                err = max(_rel(a, b) for a, b in zip(f, ref["fields"]))
                if prec == "double":
                    worst64 = max(worst64, err)
                else:
                    worst32 = max(worst32, err)
                runs += 1
    # the source column inside an interior tile whose loaded rows run past
    # the grid's last row (FP32, 64-row interior tiles, nz = 170): the TF/SF
    # corrections read the source profile for grid rows only
    for pol in ("TE", "TM"):
        sim = cases.mixed_te_sim(nx=300, nz=170, steps=160, seed=7, pol=pol, precision="single")
        sim["source"] = dict(sim["source"], ix=120)
        ref = oracle.fdtd2D(dict(sim, precision="double"), fields=True)
        ctx = Context(0)
        job = Job(sim, ctx)
        job.advance(10 ** 9)
        f = job.fields()
        job.close()
        ctx.close()
        worst32 = max(worst32, max(_rel(a, b) for a, b in zip(f, ref["fields"])))
        runs += 1
    # more than 256 materials (16-bit index), and an uneven batch of couplers
    sim = cases.mixed_te_sim(nx=200, nz=120, steps=120, seed=9)
    sim["eps"] = 1.0 + 11.0 * np.random.default_rng(1).random(sim["eps"].shape)
    ctx = Context(0)
    job = Job(sim, ctx)
    job.advance(10 ** 9)
    f = job.fields()
    job.close()
    ctx.close()
    worst64 = max(worst64, max(_rel(a, b) for a, b in zip(f, oracle.fdtd2D(sim, fields=True)["fields"])))
    outs = fdtd2D_batch(workloads.coupler_batch_sims(n=6, steps=300, precision="double"))
    runs += 2
    _lib.check(lib.orf_check_violations(C.byref(cnt), 0), "check counter")
    print(json.dumps({"violations": int(cnt.value), "runs": runs, "worst_fp64": worst64, "worst_fp32": worst32,
                      "batch_finite": bool(all(np.isfinite(o["flux"]).all() for o in outs))}))


if __name__ == "__main__":
    main()
