"""3D parity of the CUDA engine against the CPU oracle through the C ABI, and
the reference's 3D physics test (tests/TestFDTD3D.m:216-228) on the GPU."""
import numpy as np
import pytest

import oracle
import opticrcwafdtd_b200 as orf
from opticrcwafdtd_b200 import Context, Job, epsComponents3D
from tests import cases

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    nb = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0)


def gpu3(sim):
    ctx = Context(0)
    job = Job(sim, ctx, dims=3)
    job.advance(10 ** 9)
    f = job.fields()
    out = job.finish()
    job.close()
    ctx.close()
    out["fields"] = f
    return out


def compare3(out, ref, ftol=1e-10, dtol=1e-9):
    for a, b, name in zip(out["fields"], ref["fields"], ["Ex", "Ey", "Ez", "Hx", "Hy", "Hz"]):
        assert rel_l2(a, b) <= ftol, (name, rel_l2(a, b))
    s = np.max(np.abs(ref["flux"]))
    assert np.max(np.abs(out["flux"] - ref["flux"])) / s <= dtol
    for mo, mr in zip(out["mon"], ref["mon"]):
        for k in ("Ea", "Eb", "Ha", "Hb"):
            sc = max(np.max(np.abs(mr[k])), 1e-300)
            assert np.max(np.abs(mo[k] - mr[k])) / sc <= dtol, k
    assert out["steps"] == ref["steps"]


@pytest.mark.parametrize("axis,per", [(3, (False, False, False)), (1, (False, False, False)),
                                      (2, (True, False, False)), (3, (True, True, False)),
                                      (1, (False, True, True))])
def test_fp64_parity_3d(axis, per):
    sim = cases.box3d_sim(axis=axis, per=per, steps=120, seed=axis)
    ref = oracle.fdtd3D(sim, fields=True)
    compare3(gpu3(sim), ref)


def test_fp32_3d_against_fp64_oracle():
    sim = cases.box3d_sim(axis=3, steps=150, precision="single", seed=7)
    out = gpu3(sim)
    ref = oracle.fdtd3D(dict(sim, precision="double"), fields=True)
    assert np.max(np.abs(out["flux"] - ref["flux"])) / np.max(np.abs(ref["flux"])) < 1e-4
    for a, b in zip(out["fields"], ref["fields"]):
        assert rel_l2(a, b) < 1e-4


def test_3d_slab_matches_tmm():
    # tests/TestFDTD3D.m:216-228
    d = 0.01
    x = np.arange(2) * d
    y = x.copy()
    z = np.round(np.arange(0, 6 + d / 2, d), 12)
    lam = np.linspace(1.2, 1.8, 7)
    sim = cases.plane_wave_3d(x, y, z, d, lam, 1.5, 0.3, 1, 0.6, 5)
    sim["eps"] = epsComponents3D(x, y, z, 1, [])
    o0 = orf.fdtd3D(sim)
    sim["eps"] = epsComponents3D(x, y, z, 1, [["box", [-np.inf, np.inf, -np.inf, np.inf, 3, 3.5, 2]]])
    o1 = orf.fdtd3D(sim)
    R = -o1["flux"][0] / o0["flux"][1]
    T = o1["flux"][1] / o0["flux"][1]
    tm = oracle.tmm(lam, [1, 2, 1], [0.5], 0, "s")
    assert np.max(np.abs(R - tm["R"].ravel())) < 2e-3
    assert np.max(np.abs(R + T - 1)) < 2e-5
    assert np.max(np.abs(o0["flux"][0] / o0["flux"][1])) < 1e-8
    ref = oracle.fdtd3D(sim)
    assert o1["steps"] == ref["steps"]
    assert np.max(np.abs(o1["flux"] - ref["flux"])) / np.max(np.abs(ref["flux"])) < 1e-9
