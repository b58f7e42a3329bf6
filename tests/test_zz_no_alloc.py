"""orf_fdtd2d_run_noalloc: the run for callers that cannot allocate device
memory at call time (their device memory belongs to their own pool, or they
may not block on the allocator).  Its device state lives in a fixed static
array inside the library, so this checks, through the C ABI, that two calls in
a row each give the same result as the allocating orf_fdtd2d_run, and that an
oversized run is refused cleanly.  Kept in its own file, collected last."""
import ctypes as C

import numpy as np
import pytest

from opticrcwafdtd_b200 import _abi, _lib, workloads
from tests import cases

pytestmark = pytest.mark.gpu

TOL = 1e-9   # the DFT/flux tolerance of the parity tests


def _run(sim, noalloc):
    lib = _lib.load()
    m = _abi.marshal_sim2d(sim)
    o, bufs = _abi.alloc_out2d(m)
    if noalloc:
        st = lib.orf_fdtd2d_run_noalloc(C.byref(m.struct), C.byref(o), None)
    else:
        st = lib.orf_fdtd2d_run(C.byref(m.struct), C.byref(o), _abi.PROGRESS_FN(0), None)
    return st, _abi.finish_out2d(m, o, bufs)


def _same(a, b):
    for k in ("flux", "fluxZ", "P", "B", "PZ", "AZ"):
        if b[k].size:
            scale = max(np.max(np.abs(b[k])), 1e-300)
            assert np.max(np.abs(a[k] - b[k])) / scale <= TOL, k
    assert a["steps"] == b["steps"]


@pytest.mark.parametrize("make", [
    lambda: cases.mixed_te_sim(nx=300, nz=160, steps=300, seed=21),
    lambda: cases.mixed_te_sim(nx=300, nz=160, steps=300, seed=22, pol="TM", precision="single"),
    lambda: workloads.coupler_sim(steps=600),
])
def test_noalloc_matches_allocating_run_twice(make):
    sim = make()
    st, ref = _run(sim, noalloc=False)
    assert st == 0, _lib.last_error()
    for _ in range(2):
        st, out = _run(sim, noalloc=True)
        assert st == 0, _lib.last_error()
        _same(out, ref)


def test_noalloc_rejects_runs_above_its_limit():
    sim = cases.mixed_te_sim(nx=2400, nz=2000, steps=50, seed=23)   # ~230 MB of FP64 state
    st, _ = _run(sim, noalloc=True)
    assert st == 8   # ORF_ETOOLARGE
    assert "limit" in _lib.last_error()
