"""The bounds-checked build (lib/liborf_fdtd_check.so, -DORF_CHECK) stands in
for a device-side memory checker: its 2D step kernels test every global
access against the extent of its buffer and every stored cell against the
grid, count what fails and skip it.  Small runs over TE/TM, periodic z, FP32
and FP64, fused depths 3-10 with both interior variants, a source column in
an interior tile whose rows run past the grid, a 16-bit material index and an
uneven batch go through it (in a process of their own, which
loads that library); the test requires no violation and the oracle's
fields (1e-10 FP64, 1e-4 FP32)."""
import json
import os
import subprocess
import sys

import pytest

from opticrcwafdtd_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECK_LIB = os.path.join(ROOT, "opticrcwafdtd_b200", "lib", "liborf_fdtd_check.so")


@pytest.mark.gpu
def test_checked_build_counts_no_out_of_bounds_access():
    assert os.path.exists(CHECK_LIB), "build the checked library: python -m opticrcwafdtd_b200.build --check"
    env = dict(os.environ, ORF_FDTD_LIB=CHECK_LIB)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "check_build_runner.py")], env=env,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["violations"] == 0, res
    assert res["worst_fp64"] <= 1e-10 and res["worst_fp32"] <= 1e-4, res
    assert res["batch_finite"] and res["runs"] >= 36


def test_normal_build_has_no_check_counter():
    import ctypes as C
    lib = _lib.load()
    n = C.c_uint64(7)
    assert lib.orf_check_violations(C.byref(n), 0) == 1   # ORF_EINVAL
    assert n.value == 0 and "normal build" in _lib.last_error()
