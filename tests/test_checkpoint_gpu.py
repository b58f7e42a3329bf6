"""Checkpoint / resume of device-resident jobs (orf_job_checkpoint /
orf_job_restore): a run stopped between chunks, saved to host and loaded
into a new job -- on a context with another fused depth -- continues bitwise
as if it had never stopped; a run that used up its step budget continues
under a larger maxTime; checkpoints of other runs are refused."""
import numpy as np
import pytest

import opticrcwafdtd_b200 as orf
from opticrcwafdtd_b200 import Context, Job
from tests import cases

pytestmark = pytest.mark.gpu


def _run(sim, dims, stop=None, tsteps=0):
    """Uninterrupted (stop None) or stopped after `stop` steps, checkpointed,
    restored into a fresh job on a context tuned with `tsteps`, finished."""
    ctx = Context(0)
    job = Job(sim, ctx, dims=dims)
    if stop is not None:
        job.advance(stop)
        state = job.checkpoint()
        job.close()
        ctx.close()
        ctx = Context(0)
        ctx.set_tuning(tsteps=tsteps)
        job = Job(sim, ctx, dims=dims)
        job.restore(state)
    job.advance(10 ** 9)
    f = job.fields()
    out = job.finish()
    steps = job.steps
    job.close()
    ctx.close()
    return f, out, steps


def _same2d(a, b):
    for x, y in zip(a[0], b[0]):
        assert np.array_equal(x, y)
    for k in ("flux", "fluxZ", "P", "B", "PZ", "AZ"):
        assert np.array_equal(a[1][k], b[1][k]), k
    assert a[2] == b[2]


@pytest.mark.parametrize("pol,precision,periodic,tsteps", [("TE", "single", False, 4), ("TM", "double", True, 3)])
def test_2d_resume_is_bitwise(pol, precision, periodic, tsteps):
    sim = cases.mixed_te_sim(nx=260, nz=140, steps=600, precision=precision, seed=11, pol=pol, periodic=periodic)
    _same2d(_run(sim, 2), _run(sim, 2, stop=250, tsteps=tsteps))


def test_3d_resume_is_bitwise():
    sim = cases.box3d_sim(steps=300, precision="single", seed=3, axis=1)
    a = _run(sim, 3)
    b = _run(sim, 3, stop=150)
    for x, y in zip(a[0], b[0]):
        assert np.array_equal(x, y)
    assert np.array_equal(a[1]["flux"], b[1]["flux"])
    for ma, mb in zip(a[1]["mon"], b[1]["mon"]):
        for k in ("Ea", "Eb", "Ha", "Hb"):
            assert np.array_equal(ma[k], mb[k]), k
    assert a[2] == b[2]


def test_run_past_its_budget_continues_under_a_larger_one():
    short = cases.mixed_te_sim(nx=240, nz=120, steps=400, precision="single", seed=12)
    long = dict(short, maxTime=short["maxTime"] * 2.0)
    ctx = Context(0)
    job = Job(short, ctx)
    job.advance(10 ** 9)
    assert job.steps == 400
    state = job.checkpoint()
    job.close()
    job = Job(long, ctx)
    job.restore(state)
    assert job.steps == 400
    job.advance(10 ** 9)
    out, steps = job.finish(), job.steps
    job.close()
    ref = orf.fdtd2D(long, ctx)
    ctx.close()
    assert steps == ref["steps"] == 800
    for k in ("flux", "fluxZ", "P", "B"):
        assert np.array_equal(out[k], ref[k]), k


def test_checkpoint_of_another_run_is_refused():
    ctx = Context(0)
    a = Job(cases.mixed_te_sim(nx=200, nz=100, steps=200, precision="single"), ctx)
    b = Job(cases.mixed_te_sim(nx=201, nz=100, steps=200, precision="single"), ctx)
    c = Job(cases.box3d_sim(steps=100, precision="single"), ctx, dims=3)
    a.advance(100)
    state = a.checkpoint()
    for other in (b, c):
        with pytest.raises(orf.OrfError):
            other.restore(state)
    with pytest.raises(orf.OrfError):
        a.restore(state[:-1])
    a.restore(state)          # its own state loads back
    assert a.steps == 100
    for j in (a, b, c):
        j.close()
    ctx.close()
