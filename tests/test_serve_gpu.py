"""Serving loop (orf_serve_*): jobs admitted by device-memory budget, advanced
together in macro-steps, retired on shutoff or step budget.  A job's result in
a mixed stream is bitwise the result of the same sim run alone."""
import numpy as np
import pytest

import opticrcwafdtd_b200 as orf
from tests import cases

pytestmark = pytest.mark.gpu


def _bitwise2d(a, b):
    for k in ("flux", "fluxZ", "P", "B", "PZ", "AZ"):
        assert np.array_equal(a[k], b[k]), k
    assert a["steps"] == b["steps"] and a["converged"] == b["converged"]


def _bitwise3d(a, b):
    assert np.array_equal(a["flux"], b["flux"])
    for ma, mb in zip(a["mon"], b["mon"]):
        for k in ("Ea", "Eb", "Ha", "Hb"):
            assert np.array_equal(ma[k], mb[k]), k
    assert a["steps"] == b["steps"]


def _mix(precision):
    sims2 = [cases.mixed_te_sim(nx=nx, nz=nz, steps=st, seed=50 + q, precision=precision, pol=pol)
             for q, (nx, nz, st, pol) in enumerate([(300, 160, 700, "TE"), (180, 120, 450, "TE"),
                                                     (420, 140, 300, "TM"), (260, 200, 900, "TE"),
                                                     (200, 90, 250, "TM")])]
    sims3 = [cases.box3d_sim(steps=st, seed=60 + q, precision=precision, axis=ax)
             for q, (st, ax) in enumerate([(200, 3), (350, 1)])]
    return sims2, sims3


@pytest.mark.parametrize("precision", ["single", "double"])
def test_served_jobs_equal_alone_runs(precision):
    sims2, sims3 = _mix(precision)
    alone2 = [orf.fdtd2D(s) for s in sims2]
    alone3 = [orf.fdtd3D(s) for s in sims3]
    srv = orf.Server(macro_steps=100)
    # staggered arrivals: half now, the rest after two scheduling rounds
    t2 = [srv.submit(s) for s in sims2[:3]]
    t3 = [srv.submit(sims3[0], dims=3)]
    srv.step()
    srv.step()
    t2 += [srv.submit(s) for s in sims2[3:]]
    t3 += [srv.submit(sims3[1], dims=3)]
    srv.drain()
    for t, a in zip(t2, alone2):
        _bitwise2d(srv.result(t), a)
    for t, a in zip(t3, alone3):
        _bitwise3d(srv.result(t), a)
    infos = [srv.info(t) for t in t2 + t3]
    assert all(i["status"] == 0 and i["t_submit"] <= i["t_admit"] <= i["t_done"] for i in infos)
    assert [i["dims"] for i in infos] == [2] * 5 + [3] * 2
    srv.close()


def test_budget_admits_one_job_at_a_time():
    sims2, _ = _mix("single")
    a, b = sims2[0], sims2[3]
    alone_a, alone_b = orf.fdtd2D(a), orf.fdtd2D(b)
    # learn the jobs' footprints from a server with room for both
    probe = orf.Server()
    pa, pb = probe.submit(a), probe.submit(b)
    probe.drain()
    na, nb = probe.info(pa)["device_bytes"], probe.info(pb)["device_bytes"]
    probe.close()
    assert na > 0 and nb > 0
    srv = orf.Server(max_device_bytes=max(na, nb) + min(na, nb) // 2, max_jobs=8, macro_steps=50)
    ta, tb = srv.submit(a), srv.submit(b)
    srv.step()
    assert srv.pending() == (1, 1)          # the second job waits for memory
    srv.drain()
    ia, ib = srv.info(ta), srv.info(tb)
    assert ib["t_admit"] >= ia["t_done"]
    _bitwise2d(srv.result(ta), alone_a)
    _bitwise2d(srv.result(tb), alone_b)
    srv.close()


def test_job_larger_than_budget_fails_alone():
    s = cases.mixed_te_sim(nx=300, nz=160, steps=100, precision="single")
    srv = orf.Server(max_device_bytes=1 << 16)
    t = srv.submit(s)
    srv.drain()
    assert srv.info(t)["status"] == 8            # ORF_ETOOLARGE
    with pytest.raises(orf.OrfError):
        srv.result(t)
    srv.close()


def test_slot_limit_and_shutoff():
    s1 = cases.progress_sim()
    s2 = dict(cases.progress_sim(), maxTime=3.0)
    srv = orf.Server(max_jobs=1)
    t1, t2 = srv.submit(s1), srv.submit(s2)
    srv.step()
    assert srv.pending() == (1, 1)
    srv.drain()
    o1, o2 = srv.result(t1), srv.result(t2)
    assert o1["converged"] and not o2["converged"]
    assert o1["steps"] == orf.fdtd2D(s1)["steps"]
    srv.close()


def test_poll_unknown_ticket_and_busy():
    srv = orf.Server()
    with pytest.raises(orf.OrfError):
        srv.info(12345)
    t = srv.submit(cases.mixed_te_sim(steps=100, precision="single"))
    assert srv.info(t) is None
    with pytest.raises(orf.OrfError):
        srv.result(t)
    srv.drain()
    assert srv.info(t)["status"] == 0
    srv.close()


@pytest.mark.parametrize("precision", ["single", "double"])
def test_preempted_jobs_equal_alone_runs(precision):
    """Jobs preempted mid-run (their state parked in host memory, their
    device memory freed) and re-admitted later -- into groups at either
    buffer parity -- finish bitwise as when run alone."""
    sims2, sims3 = _mix(precision)
    alone2 = [orf.fdtd2D(s) for s in sims2]
    alone3 = [orf.fdtd3D(s) for s in sims3]
    srv = orf.Server(macro_steps=100)
    t2 = [srv.submit(s) for s in sims2]
    t3 = [srv.submit(s, dims=3) for s in sims3]
    srv.step()
    srv.preempt(t2[0])
    srv.preempt(t3[1])
    srv.step()
    srv.preempt(t2[3])
    srv.preempt(t2[0])          # re-admitted above, preempted again
    srv.step()
    srv.drain()
    for t, a in zip(t2, alone2):
        _bitwise2d(srv.result(t), a)
    for t, a in zip(t3, alone3):
        _bitwise3d(srv.result(t), a)
    pre = {t: srv.info(t)["preemptions"] for t in t2 + t3}
    assert pre[t2[0]] == 2 and pre[t2[3]] == 1 and pre[t3[1]] == 1
    assert sum(pre.values()) == 4
    srv.close()


def test_preemption_frees_memory_for_the_queue():
    """With room for one job, preempting the resident one lets the queued
    job run first; the preempted one resumes afterwards, both exact."""
    sims2, _ = _mix("single")
    a, b = sims2[0], sims2[3]
    alone_a, alone_b = orf.fdtd2D(a), orf.fdtd2D(b)
    probe = orf.Server()
    pa, pb = probe.submit(a), probe.submit(b)
    probe.drain()
    na, nb = probe.info(pa)["device_bytes"], probe.info(pb)["device_bytes"]
    probe.close()
    srv = orf.Server(max_device_bytes=max(na, nb) + min(na, nb) // 2, max_jobs=8, macro_steps=50)
    ta, tb = srv.submit(a), srv.submit(b)
    srv.step()
    assert srv.pending() == (1, 1)          # a resident, b waiting for memory
    srv.preempt(ta)
    assert srv.pending() == (2, 0)
    srv.step()
    assert srv.pending() == (1, 1)          # b resident now, a waits
    srv.drain()
    ia, ib = srv.info(ta), srv.info(tb)
    assert ia["preemptions"] == 1 and ib["preemptions"] == 0
    assert ia["t_done"] >= ib["t_admit"]
    _bitwise2d(srv.result(ta), alone_a)
    _bitwise2d(srv.result(tb), alone_b)
    with pytest.raises(orf.OrfError):
        srv.preempt(10 ** 6)
    srv.close()
