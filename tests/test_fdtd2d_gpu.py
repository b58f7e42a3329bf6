"""2D parity of the CUDA engine against the CPU oracle, through the C ABI.

Bars: FP64 fields <= 1e-10 relative L2, monitored flux
<= 1e-9 absolute after normalisation; FP32 + Kahan form within the
reference's single-vs-double tolerance (1e-4, tests/TestFDTD2D.m:68-74).
Physics tests of the reference are repeated on the GPU path at the
reference's tolerances."""
import numpy as np
import pytest

import oracle
import opticrcwafdtd_b200 as orf
from opticrcwafdtd_b200 import Context, Job
from tests import cases

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-10
FLUX_TOL = 1e-9


def rel_l2(a, b):
    n = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (n if n > 0 else 1.0)


def gpu_run(sim, tsteps=0, variant=0, graph=True):
    ctx = Context(0)
    ctx.set_tuning(tsteps=tsteps, variant=variant, use_graph=graph)
    job = Job(sim, ctx)
    job.advance(10 ** 9)
    f = job.fields()
    out = job.finish()
    job.close()
    ctx.close()
    out["fields"] = f
    return out


def compare(out, ref, field_tol=FIELD_TOL, flux_tol=FLUX_TOL):
    for a, b, name in zip(out["fields"], ref["fields"], "PAB"):
        assert rel_l2(a, b) <= field_tol, (name, rel_l2(a, b))
    scale = max(np.max(np.abs(ref["flux"])), 1e-300)
    assert np.max(np.abs(out["flux"] - ref["flux"])) / scale <= flux_tol
    if ref["fluxZ"].size:
        sz = max(np.max(np.abs(ref["fluxZ"])), 1e-300)
        assert np.max(np.abs(out["fluxZ"] - ref["fluxZ"])) / sz <= flux_tol
    for k in ("P", "B", "PZ", "AZ"):
        if ref[k].size:
            s = max(np.max(np.abs(ref[k])), 1e-300)
            assert np.max(np.abs(out[k] - ref[k])) / s <= flux_tol, k
    assert out["steps"] == ref["steps"]


@pytest.mark.parametrize("pol,periodic", [("TE", False), ("TM", False), ("TE", True), ("TM", True)])
def test_fp64_parity_mixed(pol, periodic):
    sim = cases.mixed_te_sim(pol=pol, periodic=periodic, steps=420)
    ref = oracle.fdtd2D(sim, fields=True)
    out = gpu_run(sim)
    compare(out, ref)


@pytest.mark.parametrize("tsteps", [1, 2, 5, 8])
@pytest.mark.parametrize("variant", [1, 2])
def test_temporal_block_depth_and_variant_invariance(tsteps, variant):
    sim = cases.mixed_te_sim(steps=333, seed=5)
    ref = oracle.fdtd2D(sim, fields=True)
    out = gpu_run(sim, tsteps=tsteps, variant=variant)
    compare(out, ref)


@pytest.mark.parametrize("precision", ["single", "double"])
@pytest.mark.parametrize("pol,periodic", [("TE", False), ("TM", False), ("TM", True)])
def test_tiling_changes_no_bit(precision, pol, periodic):
    """The fused depth T and the interior variant move cells between interior
    tiles, frame tiles of each CPML-axis specialisation and the overlap of
    neighbouring tiles; every cell performs the same roundings wherever it
    lands, so fields and DFT lines are bitwise those of the default tiling."""
    sim = cases.mixed_te_sim(nx=700, nz=330, steps=300, precision=precision, seed=5, pol=pol, periodic=periodic)
    ref = gpu_run(sim)
    for tsteps, variant in [(3, 1), (4, 1), (6, 2), (8, 2), (10, 1)]:
        out = gpu_run(sim, tsteps=tsteps, variant=variant)
        for a, b, name in zip(out["fields"], ref["fields"], "PAB"):
            assert np.array_equal(a, b), (tsteps, variant, name)
        for k in ("flux", "fluxZ", "P", "B", "PZ", "AZ"):
            assert np.array_equal(out[k], ref[k]), (tsteps, variant, k)


def test_graph_and_direct_launch_agree_bitwise():
    sim = cases.mixed_te_sim(steps=1000, seed=2)
    a = gpu_run(sim, graph=True)
    b = gpu_run(sim, graph=False)
    for x, y in zip(a["fields"], b["fields"]):
        assert np.array_equal(x, y)
    assert np.array_equal(a["flux"], b["flux"])


def test_many_materials_uses_uint16_index():
    sim = cases.mixed_te_sim(steps=200, seed=9)
    rng = np.random.default_rng(1)
    sim["eps"] = 1.0 + 11.0 * rng.random(sim["eps"].shape)   # > 256 distinct values
    ref = oracle.fdtd2D(sim, fields=True)
    compare(gpu_run(sim), ref)


def test_fp32_kahan_form_against_fp64_oracle():
    sim = cases.mixed_te_sim(steps=600, precision="single", seed=4)
    out = gpu_run(sim)
    sim64 = dict(sim, precision="double")
    ref = oracle.fdtd2D(sim64, fields=True)
    scale = np.max(np.abs(ref["flux"]))
    assert np.max(np.abs(out["flux"] - ref["flux"])) / scale < 1e-4
    for a, b in zip(out["fields"], ref["fields"]):
        assert rel_l2(a, b) < 1e-4


def test_slab_matches_tmm_on_gpu():
    # tests/TestFDTD2D.m:52-58, 136-140 on the GPU path
    R, T, Re = cases.slab_rt(orf.fdtd2DTE, 0.01)
    tm = oracle.tmm(np.linspace(1.2, 1.8, 7), [1, 2, 1], [0.5], 0, "s")
    assert np.max(np.abs(R - tm["R"].ravel())) < 3e-3
    assert np.max(np.abs(R + T - 1)) < 2e-5
    assert np.max(Re) < 1e-8
    # gpuMatchesCpu (tests/TestFDTD2D.m:76-84): GPU double vs CPU double 1e-10
    Ro, To, _ = cases.slab_rt(oracle.fdtd2DTE, 0.01)
    assert np.max(np.abs(R - Ro)) < 1e-10 and np.max(np.abs(T - To)) < 1e-10
    R3, _, _ = cases.slab_rt(orf.fdtd2DTE, 0.01, {"precision": "single"})
    assert np.max(np.abs(R3 - Ro)) < 1e-4


def test_mode_source_unidirectional_on_gpu():
    # tests/TestFDTD2D.m:142-147
    sim, _ = cases.waveguide_sim()
    o = orf.fdtd2DTE(sim)
    back = -o["flux"][0] / o["flux"][1]
    assert np.max(np.abs(back)) < 1e-4
    assert np.max(np.abs(o["flux"][2] / o["flux"][1] - 1)) < 1e-4
    ref = oracle.fdtd2DTE(sim)
    assert o["steps"] == ref["steps"]
    assert np.max(np.abs(o["flux"] - ref["flux"])) / np.max(np.abs(ref["flux"])) < FLUX_TOL


def test_tm_guided_mode_on_gpu():
    sim, _, _ = cases.waveguide_tm_sim()
    o = orf.fdtd2D(sim)
    assert -o["flux"][0, 0] / o["flux"][1, 0] < 1e-6
    assert abs(o["flux"][2, 0] / o["flux"][1, 0] - 1) < 1e-5
    ref = oracle.fdtd2D(sim)
    assert np.max(np.abs(o["Hy"] - ref["Hy"])) / np.max(np.abs(ref["Hy"])) < FLUX_TOL


def test_progress_and_cancel_on_gpu():
    # tests/TestGUISupport.m:27-45
    s = cases.progress_sim()
    fr = []
    s["progress"] = lambda f, msg: fr.append(f)
    o = orf.fdtd2DTE(s)
    assert o["converged"]
    assert len(fr) > 3 and all(0 <= f <= 1 for f in fr) and fr[-1] > 0.9
    ref = oracle.fdtd2DTE(dict(s, progress=None))
    assert o["steps"] == ref["steps"]

    class Cancelled(Exception):
        identifier = "orf:cancelled"

    def cancel_after(f, msg):
        if f > 0.2:
            raise Cancelled("stop")

    s["progress"] = cancel_after
    with pytest.raises(Cancelled):
        orf.fdtd2DTE(s)
    # the context stays usable after a cancel
    s["progress"] = None
    assert orf.fdtd2DTE(s)["converged"]


def test_not_converged_warning():
    s = cases.progress_sim()
    s["maxTime"] = 2.0
    with pytest.warns(orf.NotConvergedWarning):
        o = orf.fdtd2DTE(s)
    assert not o["converged"]


def test_job_reset_is_deterministic():
    sim = cases.mixed_te_sim(steps=300, seed=7)
    ctx = Context(0)
    job = Job(sim, ctx)
    job.advance(300)
    f1 = job.fields()
    o1 = job.finish()
    job.reset()
    job.advance(120)
    assert job.steps == 150            # whole chunks of 50 steps
    job.advance(300)
    f2 = job.fields()
    o2 = job.finish()
    for a, b in zip(f1, f2):
        assert np.array_equal(a, b)
    assert np.array_equal(o1["flux"], o2["flux"])
    job.close()
    ctx.close()


@pytest.mark.parametrize("pol,periodic,tsteps,variant", [
    ("TE", False, 6, 1), ("TM", False, 6, 1), ("TE", True, 4, 2), ("TM", False, 3, 2), ("TE", False, 1, 1),
])
def test_fp64_parity_many_interior_tiles(pol, periodic, tsteps, variant):
    """Grid large enough for dozens of pipelined interior tiles plus the CPML frame."""
    sim = cases.mixed_te_sim(nx=700, nz=330, steps=250, pol=pol, periodic=periodic, seed=11)
    ref = oracle.fdtd2D(sim, fields=True)
    compare(gpu_run(sim, tsteps=tsteps, variant=variant), ref)


def test_fp32_many_tiles_against_fp64_oracle():
    sim = cases.mixed_te_sim(nx=700, nz=330, steps=400, pol="TM", precision="single", seed=12)
    out = gpu_run(sim, tsteps=6)
    ref = oracle.fdtd2D(dict(sim, precision="double"), fields=True)
    scale = np.max(np.abs(ref["flux"]))
    assert np.max(np.abs(out["flux"] - ref["flux"])) / scale < 1e-4
    for a, b in zip(out["fields"], ref["fields"]):
        assert rel_l2(a, b) < 1e-4


@pytest.mark.parametrize("precision", ["double", "single"])
def test_partial_last_chunk_large_grid_is_finite(precision):
    """A step budget that ends inside a chunk (1344 = 26 x 50 + 44 steps) on a
    grid with tens of DFT flush blocks: every DFT line stays finite, whatever
    shared memory held before (the flush weights steps past the budget by
    exact zeros), and FP32 agrees with FP64."""
    from opticrcwafdtd_b200 import workloads
    sim = workloads._coupler_instance(3213, 1071, 0.63, 0.5, 0.07, 1344, precision, 21)
    out = orf.fdtd2D(sim)
    for k in ("flux", "fluxZ", "P", "B", "PZ", "AZ"):
        assert np.isfinite(out[k]).all(), k
    assert out["steps"] == 1344
    if precision == "single":
        ref = orf.fdtd2D(dict(sim, precision="double"))
        assert np.max(np.abs(out["flux"] - ref["flux"])) / np.max(np.abs(ref["flux"])) < 1e-4


def test_context_may_be_released_before_its_job_and_server():
    """Jobs and servers hold a reference to their context: releasing the
    context first (as a garbage collector may do) leaves them working."""
    sim = cases.mixed_te_sim(nx=200, nz=100, steps=150, precision="single")
    ref = orf.fdtd2D(sim)
    ctx = Context(0)
    job = Job(sim, ctx)
    srv = orf.Server(ctx)
    ctx.close()
    job.advance(150)
    out = job.finish()
    job.close()
    t = srv.submit(sim)
    srv.drain()
    assert np.array_equal(srv.result(t)["flux"], ref["flux"])
    assert np.array_equal(out["flux"], ref["flux"])
    srv.close()
