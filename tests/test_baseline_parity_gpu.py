"""FP64 parity with the oracle on the benchmark configurations themselves,
at their full grid sizes (the other parity tests use small grids).

  C1  2D TE SOI grating coupler, 800 x 300, FP64, all 8000 steps: the
      drop-in correctness case (tests/TestFDTD2D.m:76-84: GPU against CPU
      within 1e-10);
  C2  2D TM Si/SiO2 pixel region, 4000 x 1500, FP64, 2000 of its 30000 steps;
  C3  3D TiO2 pillar lattice, 600 x 600 x 300, FP64, 60 of its 6000 steps;
  C4  256 uneven grating couplers in FP32 through one orf_batch2d_run: the
      fiber coupling efficiency (fiberCoupling.m:16-31) of 8 seeded
      instances within 1e-3 absolute of the FP64 oracle (tests/TestCPO.m:26-34
      reads the same budget).

Bars: fields within 1e-10 relative L2; every DFT line within 1e-9 of its
largest magnitude (3D: of the plane's largest E or H); the monitored transmission T = flux / incident flux
within 1e-9 absolute.  Where the run covers the whole pulse (C1, C4) the
incident flux is the one through the monitor just after the source, per
wavelength; C2 and C3 stop on the rising edge of the pulse, where a
wavelength's incident flux may pass through zero, so there T is taken
against the largest incident flux over the wavelengths (C3: over its
monitors too; after 60 steps only the plane behind the source, at 10 cells,
and the first plane past the pillars, at 55, lie inside the light cone of
the source, and a plane outside it must read exactly zero on both sides)."""
import warnings

import numpy as np
import pytest

import oracle
from opticrcwafdtd_b200 import Context, Job, fdtd2D_batch, workloads

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

FIELD_TOL = 1e-10
LINE_TOL = 1e-9
T_TOL = 1e-9
ETA_TOL = 1e-3


def _rel_l2(a, b):
    n = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (n if n > 0 else 1.0)


def _gpu(sim, dims):
    ctx = Context(0)
    job = Job(sim, ctx, dims=dims)
    job.advance(10 ** 9)
    f = job.fields()
    out = job.finish()
    job.close()
    ctx.close()
    out["fields"] = f
    return out


def _oracle(sim, dims):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return oracle.fdtd2D(sim, fields=True) if dims == 2 else oracle.fdtd3D(sim, fields=True)


def _check_lines(out, ref, keys):
    for k in keys:
        if np.size(ref[k]):
            s = max(np.max(np.abs(ref[k])), 1e-300)
            err = np.max(np.abs(out[k] - ref[k])) / s
            assert err <= LINE_TOL, (k, err)


def _check_transmission(out, ref, inc, keys=("flux", "fluxZ")):
    assert np.all(np.abs(inc) > 0)
    for k in keys:
        if np.size(ref[k]):
            err = np.max(np.abs(out[k] / inc - ref[k] / inc))
            assert err <= T_TOL, (k, err)


def test_c1_coupler_fp64_all_steps():
    sim = workloads.coupler_sim(precision="double", steps=8000)
    assert sim["eps"].shape == (800, 300)
    ref = _oracle(sim, 2)
    out = _gpu(sim, 2)
    assert out["steps"] == ref["steps"] == 8000
    for a, b, name in zip(out["fields"], ref["fields"], "PAB"):
        assert _rel_l2(a, b) <= FIELD_TOL, (name, _rel_l2(a, b))
    _check_lines(out, ref, ("P", "B", "PZ", "AZ"))
    # incident flux per wavelength: the line just after the source (monitor 2)
    _check_transmission(out, ref, ref["flux"][1][None, :])


def test_c2_pixel_region_fp64_full_grid():
    sim = workloads.pixel_region_sim(precision="double", steps=2000)
    assert sim["epsX"].shape[0] == 4000 and sim["epsZ"].shape[1] == 1500
    ref = _oracle(sim, 2)
    out = _gpu(sim, 2)
    assert out["steps"] == ref["steps"] == 2000
    for a, b, name in zip(out["fields"], ref["fields"], "PAB"):
        assert np.max(np.abs(b)) > 0
        assert _rel_l2(a, b) <= FIELD_TOL, (name, _rel_l2(a, b))
    _check_lines(out, ref, ("P", "B", "PZ", "AZ"))
    _check_transmission(out, ref, np.max(np.abs(ref["flux"][1])))


def test_c3_pillar_lattice_fp64_full_grid():
    sim = workloads.pillar_lattice_sim(steps=60, precision="double", n_lambda=3, device=True)
    assert (sim["x"].size, sim["y"].size, sim["z"].size) == (600, 600, 300)
    ref = _oracle(sim, 3)
    out = _gpu(sim, 3)
    assert out["steps"] == ref["steps"] == 60
    for q in range(6):
        a, b = out["fields"].pop(0), ref["fields"].pop(0)
        assert _rel_l2(a, b) <= FIELD_TOL, ("EH"[q // 3] + "xyz"[q % 3], _rel_l2(a, b))
        del a, b
    # each plane's E lines against the plane's largest E, its H lines against
    # its largest H: a component that vanishes by symmetry on a plane (Ey of
    # the x-polarised wave behind the source reads 1e-18 of Ex, rounding
    # noise that a 1e-15 change of the source amplitude moves by its own
    # size) is compared on the scale of the field there
    for mo, mr in zip(out["mon"], ref["mon"]):
        for pair in (("Ea", "Eb"), ("Ha", "Hb")):
            s = max(max(np.max(np.abs(mr[k])) for k in pair), 1e-300)
            for k in pair:
                err = np.max(np.abs(mo[k] - mr[k])) / s
                assert err <= LINE_TOL, (k, err)
    _check_transmission(out, ref, np.max(np.abs(ref["flux"])), keys=("flux",))


def test_c4_batch_fp32_coupling_efficiency_against_fp64_oracle():
    sims = workloads.coupler_batch_sims(n=256, steps=10000, precision="single")
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        outs = fdtd2D_batch(sims)
    pick = np.unique(np.linspace(0, 255, 8).round().astype(int))
    assert pick.size == 8
    for q in pick:
        s64 = dict(sims[q], precision="double")
        ref = _oracle(s64, 2)
        assert outs[q]["steps"] == ref["steps"] == 10000
        e32, e64 = workloads.coupler_instance_eta(outs[q], sims[q]), workloads.coupler_instance_eta(ref, s64)
        assert np.max(e64) > 0.05          # a coupler, not an empty run
        err = np.max(np.abs(e32 - e64))
        assert err <= ETA_TOL, (int(q), err)
