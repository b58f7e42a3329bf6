"""Batched 2D runs (orf_batch2d_run): every instance of a batch gives the same
result as the same sim run alone, and matches the oracle."""
import numpy as np
import pytest

import oracle
import opticrcwafdtd_b200 as orf
from tests import cases

pytestmark = pytest.mark.gpu


def _same(a, b, tol):
    for k in ("flux", "fluxZ", "P", "B", "PZ", "AZ"):
        if b[k].size:
            s = max(np.max(np.abs(b[k])), 1e-300)
            assert np.max(np.abs(a[k] - b[k])) / s <= tol, k
    assert a["steps"] == b["steps"]


@pytest.mark.parametrize("precision", ["double", "single"])
def test_batch_of_uneven_instances_matches_single_runs(precision):
    sims = []
    for q, (nx, nz, steps) in enumerate([(300, 160, 300), (180, 120, 450), (420, 140, 200), (260, 200, 350)]):
        s = cases.mixed_te_sim(nx=nx, nz=nz, steps=steps, seed=30 + q, precision=precision)
        sims.append(s)
    outs = orf.fdtd2D_batch(sims)
    for s, o in zip(sims, outs):
        alone = orf.fdtd2D(s)
        _same(o, alone, 0.0 if precision == "double" else 0.0)   # same kernels, same arithmetic: bitwise
        if precision == "double":
            _same(o, oracle.fdtd2D(s), 1e-9)


def test_batch_shutoff_stops_each_instance():
    s1 = cases.progress_sim()
    s2 = dict(cases.progress_sim(), maxTime=3.0)
    o = orf.fdtd2D_batch([s1, s2])
    assert o[0]["converged"] and not o[1]["converged"]
    ref = oracle.fdtd2DTE(s1)
    assert o[0]["steps"] == ref["steps"]


def test_autotune_changes_speed_not_results():
    """orf_autotune2d picks one of the timed candidates; every candidate
    computes the same values, so tuned runs equal default runs bitwise."""
    sim = cases.mixed_te_sim(nx=700, nz=330, steps=300, precision="single", seed=5, pol="TM")
    ref = orf.fdtd2D(sim)
    ctx = orf.Context(0)
    t = ctx.autotune2d(sim, steps=100)
    assert t["variant"] in (1, 2) and t["tsteps"] in (4, 6, 8, 10) and t["use_graph"]
    out = orf.fdtd2D(sim, ctx)
    for k in ("flux", "fluxZ", "P", "B", "PZ", "AZ"):
        assert np.array_equal(out[k], ref[k]), k
    sims = [sim, cases.mixed_te_sim(nx=300, nz=160, steps=200, precision="single", seed=6, pol="TM")]
    outs = orf.fdtd2D_batch(sims, ctx, autotune=True)
    for s, o in zip(sims, outs):
        a = orf.fdtd2D(s)
        assert np.array_equal(o["flux"], a["flux"]) and np.array_equal(o["P"], a["P"])
    ctx.close()
