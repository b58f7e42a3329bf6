"""A 3D run split into z slabs (orf_job3d_create_slab + orf_job3d_step, ghost
planes swapped after every step) against the same run on one grid: own
planes of the fields, DFT monitor planes and z-normal fluxes bit for bit,
fluxes of monitor planes cut between slabs to 1e-12 (summed on the host),
in FP64 and FP32; the cut's validation through the C-ABI."""
import ctypes as C

import numpy as np
import pytest

from opticrcwafdtd_b200 import Context, Job, slab3d
from opticrcwafdtd_b200 import _abi, _lib
from tests import cases

pytestmark = pytest.mark.gpu


def _whole(sim):
    ctx = Context(0)
    job = Job(sim, ctx, dims=3)
    job.advance(10 ** 9)
    f = job.fields()
    o = job.finish()
    job.close()
    ctx.close()
    return f, o


def _compare(sim, nslabs):
    f_ref, o_ref = _whole(sim)
    out, jobs, ctx = slab3d.fdtd3D_slabs(sim, nslabs, return_jobs=True)
    try:
        own = [slab3d.own_fields(j) for j in jobs]
        for q in range(6):
            got = np.concatenate([o[q] for o in own], axis=2)
            assert got.shape == f_ref[q].shape
            bad = np.argwhere(got != f_ref[q])
            assert bad.size == 0, f"field {q}: {len(bad)} cells differ, first at {bad[0]}"
    finally:
        for j in jobs:
            j.close()
        ctx.close()
    assert out["steps"] == o_ref["steps"] and out["steps"] > 0
    mons = sim["monitors"]
    for m, mq in enumerate(mons):
        for k in ("Ea", "Eb", "Ha", "Hb"):
            assert np.array_equal(out["mon"][m][k], o_ref["mon"][m][k]), (m, k)
        if mq["axis"] == 3:
            assert np.array_equal(out["flux"][m], o_ref["flux"][m])
        else:
            np.testing.assert_allclose(out["flux"][m], o_ref["flux"][m], rtol=1e-12,
                                       atol=1e-12 * np.abs(o_ref["flux"][m]).max())
    assert np.abs(o_ref["flux"]).max() > 0


@pytest.mark.parametrize("prec", ["double", "single"])
def test_two_slabs_equal_the_single_grid(prec):
    sim = cases.box3d_sim(n=(28, 24, 40), axis=3, steps=140, precision=prec, seed=3, npml=(6, 5, 7))
    _compare(sim, 2)


@pytest.mark.parametrize("prec", ["double", "single"])
def test_three_slabs_periodic_xy_equal_the_single_grid(prec):
    sim = cases.box3d_sim(n=(32, 24, 66), axis=3, per=(True, True, False), steps=160, precision=prec, seed=4,
                          npml=(6, 5, 8))
    _compare(sim, 3)


def test_source_plane_on_the_cut():
    sim = cases.box3d_sim(n=(24, 20, 40), axis=3, steps=120, precision="double", seed=5, npml=(5, 5, 7))
    b = slab3d.split_z(40, 2, 7)[1].z0
    sim["source"]["index"] = b + 1          # E plane b (slab 1's first), H plane b-1 (slab 0's last)
    _compare(sim, 2)


def test_x_normal_source_cut_between_slabs():
    sim = cases.box3d_sim(n=(26, 20, 44), axis=1, steps=120, precision="double", seed=6, npml=(6, 5, 7))
    _compare(sim, 2)


def test_one_slab_is_the_whole_grid():
    sim = cases.box3d_sim(n=(20, 18, 30), axis=3, steps=80, precision="single", seed=7, npml=(4, 4, 6))
    _compare(sim, 1)


def test_slab_validation_through_the_c_abi():
    lib = _lib.load()
    sim = cases.box3d_sim(n=(20, 18, 40), axis=3, steps=20, precision="double", seed=8, npml=(4, 4, 7))
    ctx = Context(0)
    try:
        def create(lo, hi, **upd):
            s = dict(sim)
            s.update(upd)
            loc = slab3d.slab_sim(s, slab3d.Slab(0, lo, hi, lo, hi))
            loc["shutoff"] = upd.get("shutoff", 0.0)
            m = _abi.marshal_sim3d(loc)
            h = C.c_void_p()
            st = lib.orf_job3d_create_slab(ctx.handle, C.byref(m.struct), lo, 40, C.byref(h))
            if st == 0:
                lib.orf_job_destroy(h)
            return st, _lib.last_error()
        assert create(0, 21)[0] == 0
        st, msg = create(5, 40)              # inner end at plane 5: inside the 7-plane layer
        assert st != 0 and "CPML" in msg
        st, msg = create(0, 36)              # inner end at 36: within reach of the top layer
        assert st != 0 and "CPML" in msg
        st, msg = create(0, 21, shutoff=1e-8)
        assert st != 0 and "shutoff" in msg
        st, msg = create(30, 50)
        assert st != 0
    finally:
        ctx.close()
