"""orf_fdtd2d_run_noalloc: the run for callers that cannot allocate device
memory at call time (their device memory belongs to their own pool, or they
may not block on the allocator).  Its device state lives in a fixed static
array inside the library, so this checks, through the C ABI, that two calls in
a row each give bitwise the result of the allocating orf_fdtd2d_run (the same
kernels, the same launch order of the chunks), that after the first call on
the device no further call changes the device's free memory, and that an
oversized run is refused cleanly.  Kept in its own file, collected last."""
import ctypes as C

import numpy as np
import pytest

from opticrcwafdtd_b200 import _abi, _lib, workloads
from tests import cases

pytestmark = pytest.mark.gpu


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
        assert np.array_equal(a[k], b[k]), k
    assert a["steps"] == b["steps"]
    assert a["converged"] == b["converged"]


def _free_bytes():
    import torch
    return torch.cuda.mem_get_info(0)[0]


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


def test_noalloc_takes_no_device_memory_after_the_first_call():
    sim = cases.mixed_te_sim(nx=300, nz=160, steps=300, seed=24)
    st, first = _run(sim, noalloc=True)        # the one-time set-up on this device
    assert st == 0, _lib.last_error()
    free0 = _free_bytes()
    for _ in range(2):
        st, out = _run(sim, noalloc=True)
        assert st == 0, _lib.last_error()
        _same(out, first)
    assert _free_bytes() == free0


def test_noalloc_rejects_runs_above_its_limit():
    sim = cases.mixed_te_sim(nx=2400, nz=2000, steps=50, seed=23)   # ~230 MB of FP64 state
    st, _ = _run(sim, noalloc=True)
    assert st == 8   # ORF_ETOOLARGE
    assert "limit" in _lib.last_error()
