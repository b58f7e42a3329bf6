"""Failure detection of the 3D kernel's bounded device waits, without a GPU
fault.  The kernel's only device-side waits are the mbarrier polls of its TMA
plane ring; each gives up after a time limit, and the run then reports
ORF_ETIMEOUT_DEVICE.  The test hook of orf_ctx_set_wait_injection arms one
ring slot of every TMA tile without issuing its copies, so that wait runs out
(a flag that nothing sets).  Checked: the run returns the timeout status with
a message naming the wait, quickly; nothing faults or hangs; and the next run
on the same context is bitwise the run of a fresh context and matches the
oracle."""
import time
import warnings

import numpy as np
import pytest

import oracle
from opticrcwafdtd_b200 import Context, Job, _abi, _lib
from tests import cases

pytestmark = pytest.mark.gpu


def _sim():
    # no periodic axis: every tile loads its planes by TMA; z segments of
    # more than three planes, so the stalled plane k0 + 2 exists in each
    return cases.box3d_sim(n=(70, 40, 72), per=(False, False, False), steps=120, seed=3)


def _run(ctx, sim):
    job = Job(sim, ctx, dims=3)
    try:
        job.advance(10 ** 9)
        f = job.fields()
        out = job.finish()
    finally:
        job.close()
    out["fields"] = f
    return out


def test_stalled_plane_wait_times_out_and_context_stays_usable():
    sim = _sim()
    ctx = Context(0)
    ctx.set_wait_injection(stall_plane=2, wait_ns=2_000_000)   # 2 ms per wait
    t0 = time.perf_counter()
    with pytest.raises(_abi.OrfError) as ei:
        _run(ctx, sim)
    dt = time.perf_counter() - t0
    assert ei.value.identifier == "orf:deviceTimeout"
    assert "gave up waiting" in _lib.last_error()
    assert dt < 30.0
    # the same context, hook off: bitwise the run of a fresh context
    ctx.set_wait_injection(stall_plane=-1, wait_ns=0)
    again = _run(ctx, sim)
    ctx.close()
    fresh_ctx = Context(0)
    fresh = _run(fresh_ctx, sim)
    fresh_ctx.close()
    for a, b in zip(again["fields"], fresh["fields"]):
        assert np.array_equal(a, b)
    assert np.array_equal(again["flux"], fresh["flux"])
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        ref = oracle.fdtd3D(sim, fields=True)
    for a, b in zip(again["fields"], ref["fields"]):
        assert np.linalg.norm(a - b) <= 1e-10 * np.linalg.norm(b)


def test_wait_injection_rejects_negative_limit():
    ctx = Context(0)
    with pytest.raises(_abi.OrfError):
        ctx.set_wait_injection(stall_plane=-1, wait_ns=-5)
    ctx.close()
