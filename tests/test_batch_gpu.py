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
