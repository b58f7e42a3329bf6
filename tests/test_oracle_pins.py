"""Pins the CPU oracle against the reference's own FDTD tests, at the
reference's tolerances.  The reference's implementation is closed P-code
(toolbox/+orf/fdtd2D.p) and cannot run here, and the reference stores no
golden vectors, so these physics checks (TMM slab R/T, exact-Yee dispersion,
unidirectional source, empty-domain reflection, single vs double) are what
ties the oracle to it."""
import numpy as np
import pytest

import oracle
from tests import cases


def test_slab_matches_tmm():
    # tests/TestFDTD2D.m:52-58
    R, T, _ = cases.slab_rt(oracle.fdtd2DTE, 0.01)
    tm = oracle.tmm(np.linspace(1.2, 1.8, 7), [1, 2, 1], [0.5], 0, "s")
    assert np.max(np.abs(R - tm["R"].ravel())) < 3e-3
    assert np.max(np.abs(T - tm["T"].ravel())) < 3e-3
    assert np.max(np.abs(R + T - 1)) < 2e-5


def test_slab_error_is_second_order():
    # tests/TestFDTD2D.m:60-66
    tm = oracle.tmm(np.linspace(1.2, 1.8, 7), [1, 2, 1], [0.5], 0, "s")["R"].ravel()
    R1, _, _ = cases.slab_rt(oracle.fdtd2DTE, 0.01)
    R2, _, _ = cases.slab_rt(oracle.fdtd2DTE, 0.005)
    assert np.max(np.abs(R1 - tm)) / np.max(np.abs(R2 - tm)) > 3


def test_single_precision_matches_double():
    # tests/TestFDTD2D.m:68-74
    R1, T1, _ = cases.slab_rt(oracle.fdtd2DTE, 0.01)
    R2, T2, _ = cases.slab_rt(oracle.fdtd2DTE, 0.01, {"precision": "single"})
    assert np.max(np.abs(R2 - R1)) < 1e-4 and np.max(np.abs(T2 - T1)) < 1e-4


def test_empty_domain_has_no_reflection():
    # tests/TestFDTD2D.m:136-140
    _, _, Re = cases.slab_rt(oracle.fdtd2DTE, 0.01)
    assert np.max(Re) < 1e-8


def test_tm_slab_matches_tmm():
    # tests/TestFDTD2D.m:99-113
    from opticrcwafdtd_b200 import epsComponents2D
    dx = 0.01
    x = np.round(np.arange(0, 6 + dx / 2, dx), 12)
    z = np.arange(4) * dx
    lam = np.linspace(1.2, 1.8, 7)
    ixOf = lambda xx: int(round(xx / dx)) + 1
    s = dict(pol="TM", x=x, z=z, npml=[20, 0], periodicZ=True, lambdas=lam, monitors=[ixOf(0.6), ixOf(5)])
    s["source"] = dict(ix=ixOf(1), profile=np.ones(4), neff=1, lambda0=1.5, bw=0.3)
    e0 = epsComponents2D(x, z, 1, np.zeros((0, 5)), PeriodicZ=True)
    s["epsX"], s["epsZ"] = e0["x"], e0["z"]
    o0 = oracle.fdtd2D(s)
    e1 = epsComponents2D(x, z, 1, [3, 3.5, -np.inf, np.inf, 2], PeriodicZ=True)
    s["epsX"], s["epsZ"] = e1["x"], e1["z"]
    o1 = oracle.fdtd2D(s)
    R = -o1["flux"][0] / o0["flux"][1]
    T = o1["flux"][1] / o0["flux"][1]
    tm = oracle.tmm(lam, [1, 2, 1], [0.5], 0, "p")
    assert np.max(np.abs(R - tm["R"].ravel())) < 2e-3
    assert np.max(np.abs(R + T - 1)) < 2e-5


def _neff_from_phase(o_field, prof, k0, L, nPred):
    ph = np.angle(prof @ o_field[1]) - np.angle(prof @ o_field[0])
    q = np.round((nPred * k0 * L - ph) / (2 * np.pi))
    return (ph + 2 * np.pi * q) / (k0 * L)


def test_mode_source_unidirectional_and_dispersion():
    # tests/TestFDTD2D.m:142-165
    from opticrcwafdtd_b200 import slabModes
    sim, m = cases.waveguide_sim()
    o = oracle.fdtd2DTE(sim)
    back = -o["flux"][0] / o["flux"][1]
    assert np.max(np.abs(back)) < 1e-4
    assert np.max(np.abs(o["flux"][2] / o["flux"][1] - 1)) < 1e-4
    dx = 0.02
    S = 0.99 / np.sqrt(2) * dx
    k0 = 2 * np.pi / 1.55
    k0num = 2 / S * np.sin(k0 * S / 2)
    mt = slabModes(sim["z"], np.sqrt(sim["eps"][0, :]), 2 * np.pi / k0num, "TE")
    nPred = 2 / dx * np.arcsin(mt["neff"][0] * k0num * dx / 2) / k0
    L = (301 - 151) * dx
    f = m["field"][:, 0]
    nF = _neff_from_phase([o["Ey"][:, 2, 1], o["Ey"][:, 2, 2]], f, k0, L, nPred)
    assert abs(nF - nPred) < 2e-5


def test_tm_guided_mode_discrete_dispersion():
    # tests/TestFDTD2D.m:115-134
    from opticrcwafdtd_b200 import slabModes
    sim, m, e = cases.waveguide_tm_sim()
    o = oracle.fdtd2D(sim)
    assert -o["flux"][0, 0] / o["flux"][1, 0] < 1e-6
    assert abs(o["flux"][2, 0] / o["flux"][1, 0] - 1) < 1e-5
    dx = 0.02
    S = 0.99 / np.sqrt(2) * dx
    k0 = 2 * np.pi / 1.55
    k0n = 2 / S * np.sin(k0 * S / 2)
    mt = slabModes(sim["z"], np.sqrt(e["z"][0, :]), 2 * np.pi / k0n, "TM", EpsHalf=e["x"][0, :])
    nPred = 2 / dx * np.arcsin(mt["neff"][0] * k0n * dx / 2) / k0
    nF = _neff_from_phase([o["Hy"][:, 0, 1], o["Hy"][:, 0, 2]], m["field"][:, 0], k0, 3.0, nPred)
    assert abs(nF - nPred) < 2e-5


def test_progress_and_cancel():
    # tests/TestGUISupport.m:27-45
    s = cases.progress_sim()
    fr = []
    s["progress"] = lambda f, msg: fr.append(f)
    o = oracle.fdtd2DTE(s)
    assert o["converged"]
    assert len(fr) > 3 and all(0 <= f <= 1 for f in fr) and fr[-1] > 0.9

    class Cancelled(Exception):
        identifier = "orf:cancelled"

    def cancel_after(f, msg):
        if f > 0.2:
            raise Cancelled("stop")

    s["progress"] = cancel_after
    with pytest.raises(Cancelled):
        oracle.fdtd2DTE(s)


def test_pulse_definition():
    # g(t) = exp(-((t-t0)/tau)^2) sin(k0 (t-t0)), tau = 2/(bw k0), t0 = 5 tau
    lam, bw = 1.5, 0.3
    k0 = 2 * np.pi / lam
    tau = 2 / (bw * k0)
    for t in (0.3 * tau, 5 * tau + 0.1, 9.7 * tau):
        u = (t - 5 * tau) / tau
        assert abs(oracle.pulse(lam, bw, t) - np.exp(-u * u) * np.sin(k0 * (t - 5 * tau))) < 1e-15
    assert oracle.pulse(lam, bw, -1.0) == 0.0 and oracle.pulse(lam, bw, 10.01 * tau) == 0.0


def test_3d_slab_matches_tmm_oracle():
    # tests/TestFDTD3D.m:216-228 on the oracle
    from opticrcwafdtd_b200 import epsComponents3D
    d = 0.01
    x = np.arange(2) * d
    y = x.copy()
    z = np.round(np.arange(0, 6 + d / 2, d), 12)
    lam = np.linspace(1.2, 1.8, 7)
    sim = cases.plane_wave_3d(x, y, z, d, lam, 1.5, 0.3, 1, 0.6, 5)
    sim["eps"] = epsComponents3D(x, y, z, 1, [])
    o0 = oracle.fdtd3D(sim)
    sim["eps"] = epsComponents3D(x, y, z, 1, [["box", [-np.inf, np.inf, -np.inf, np.inf, 3, 3.5, 2]]])
    o1 = oracle.fdtd3D(sim)
    R = -o1["flux"][0] / o0["flux"][1]
    T = o1["flux"][1] / o0["flux"][1]
    tm = oracle.tmm(lam, [1, 2, 1], [0.5], 0, "s")
    assert np.max(np.abs(R - tm["R"].ravel())) < 2e-3
    assert np.max(np.abs(R + T - 1)) < 2e-5
    assert np.max(np.abs(o0["flux"][0] / o0["flux"][1])) < 1e-8


def test_3d_strip_mode_source_and_dispersion():
    """The oracle fed by wgModes2D's TE0 mode of an SOI strip: unidirectional,
    lossless, and the exact-Yee dispersion of the solved index
    (tests/TestFDTD3D.m:100-117)."""
    sim, prof, ms_eps = cases.strip3d_sim()
    cases.check_strip3d(oracle.fdtd3D(sim), sim, prof, ms_eps)
