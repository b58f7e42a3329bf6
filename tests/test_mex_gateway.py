"""The MATLAB MEX gateway (opticrcwafdtd_b200/matlab/orf_fdtd_mex.c), compiled
against the project-written mex.h / matrix.h stand-in in tests/mex_shim
(MATLAB is unavailable on this box, so the gateway is unverified with MATLAB
itself).  The sim structs are built as MATLAB would hold them: column-major
doubles, char text, logical flags, struct arrays, 1-based indices.

CPU: the orf_sim2d / orf_sim3d the gateway marshals equals, field for field,
the one the Python binding marshals (_abi.marshal_sim2d / marshal_sim3d) for
the same sim, the reference's defaults included (fdtd2D.m:9-23,
fdtd2DTE.m:7-25, fdtd3D.m:11-24); malformed sims raise orf:invalidInput, and
a valid run on a host without a GPU raises orf:noDevice.
GPU: runs through the gateway equal the Python binding's bitwise, with the
TE/TM aliases and their physical signs (fdtd2D.m:26-27), the
fdtd2D:notConverged warning, and an error thrown by the progress callback
rethrown unchanged as orf:cancelled (tests/TestGUISupport.m:39-43)."""
import math
import warnings

import numpy as np
import pytest

import opticrcwafdtd_b200 as orf
from opticrcwafdtd_b200 import _abi
from tests import cases, mexshim


@pytest.fixture(scope="module")
def gw(tmp_path_factory):
    return mexshim.Gateway(mexshim.build(str(tmp_path_factory.mktemp("mex"))))


def _py2d(sim):
    m = _abi.marshal_sim2d(sim)          # holds the arrays the struct points to
    s = m.struct
    nx, nz = s.nx, s.nz
    nzA = nz if s.periodic_z else nz - 1
    eps = np.asarray(sim.get("eps", np.zeros(1)), dtype=float)
    return {
        "pol": s.pol, "nx": nx, "nz": nz, "x0": s.x0, "z0": s.z0, "dx": s.dx, "npml_x": s.npml_x,
        "npml_z": s.npml_z, "periodic_z": s.periodic_z, "src_ix": s.src_ix, "src_neff": s.src_neff,
        "src_lambda0": s.src_lambda0, "src_bw": s.src_bw,
        "monitors": [s.monitors[i] for i in range(s.n_mon)],
        "monitors_z": [s.monitors_z[i] for i in range(s.n_monz)],
        "lambdas": [s.lambdas[i] for i in range(s.n_lambda)], "max_time": s.max_time, "shutoff": s.shutoff,
        "courant": s.courant, "precision": s.precision,
        "eps_sum": float(np.sum(eps)) if s.pol == 0 else 0.0,
        "eps_x_sum": float(np.sum(sim["epsX"])) if s.pol == 1 else 0.0,
        "eps_z_sum": float(np.sum(sim["epsZ"])) if s.pol == 1 else 0.0,
        "src_profile": [s.src_profile[k] for k in range(nz)], "_nzA": nzA, "_keep": m,
    }


def _same2d(mex, py):
    for k, v in py.items():
        if k.startswith("_"):
            continue
        m = np.atleast_1d(np.asarray(mex[k], dtype=float)).ravel()
        p = np.atleast_1d(np.asarray(v, dtype=float)).ravel()
        assert m.shape == p.shape, k
        if k.endswith("_sum"):
            np.testing.assert_allclose(m, p, rtol=1e-12, err_msg=k)
        else:
            assert np.array_equal(m, p), (k, m, p)


@pytest.mark.parametrize("make", [
    lambda: cases.mixed_te_sim(seed=3),
    lambda: cases.mixed_te_sim(seed=4, pol="TM"),
    lambda: cases.mixed_te_sim(seed=5, pol="TM", periodic=True, precision="single"),
    lambda: cases.waveguide_sim()[0],
])
def test_marshal2d_matches_python_binding(gw, make):
    sim = make()
    mex, w = gw.call("marshal2d", sim)
    assert w is None
    _same2d(mex, _py2d(sim))


def test_marshal2d_defaults_of_the_reference(gw):
    nx, nz = 60, 40
    sim = dict(x=np.arange(nx) * 0.02, z=np.arange(nz) * 0.02, eps=np.full((nx, nz), 2.25), lambdas=[1.55],
               source=dict(ix=20, profile=np.ones(nz), lambda0=1.55))
    mex, _ = gw.call("marshal2d", sim)
    _same2d(mex, _py2d(sim))
    assert mex["pol"] == 0 and mex["precision"] == 0 and mex["periodic_z"] == 0
    assert mex["npml_x"] == 0 and mex["npml_z"] == 0
    assert mex["src_neff"] == 1.0 and mex["src_bw"] == 0.2 and mex["src_ix"] == 19
    assert mex["max_time"] == 1e4 and mex["shutoff"] == 1e-10 and mex["courant"] == 0.99 / math.sqrt(2)
    # text is case-insensitive, as the wrappers pass it (char)
    mex, _ = gw.call("marshal2d", dict(sim, pol="te", precision="SINGLE"))
    assert mex["pol"] == 0 and mex["precision"] == 1


def _py3d(sim):
    mm = _abi.marshal_sim3d(sim)         # holds the arrays the struct points to
    s = mm.struct
    n = (s.nx, s.ny, s.nz)
    a, b = n[(s.src_axis + 1) % 3], n[(s.src_axis + 2) % 3]
    prof = []
    for p in (s.src_Ea, s.src_Eb, s.src_Ha, s.src_Hb):
        prof.append(float(np.sum(np.ctypeslib.as_array(p, shape=(a * b,)))))
    return {
        "nx": s.nx, "ny": s.ny, "nz": s.nz, "x0": s.x0, "y0": s.y0, "z0": s.z0, "d": s.d,
        "npml": list(s.npml), "periodic": list(s.periodic), "src_axis": s.src_axis, "src_index": s.src_index,
        "src_neff": s.src_neff, "src_lambda0": s.src_lambda0, "src_bw": s.src_bw,
        "mon_axis": [s.mon_axis[i] for i in range(s.n_mon)], "mon_index": [s.mon_index[i] for i in range(s.n_mon)],
        "lambdas": [s.lambdas[i] for i in range(s.n_lambda)], "max_time": s.max_time, "shutoff": s.shutoff,
        "courant": s.courant, "precision": s.precision,
        "eps_sums": [float(np.sum(sim["eps"][c])) for c in "xyz"], "src_sums": prof, "_keep": mm,
    }


def _same3d(mex, py):
    for k, v in py.items():
        if k.startswith("_"):
            continue
        m = np.atleast_1d(np.asarray(mex[k], dtype=float)).ravel()
        p = np.atleast_1d(np.asarray(v, dtype=float)).ravel()
        assert m.shape == p.shape, k
        if k.endswith("_sums"):
            np.testing.assert_allclose(m, p, rtol=1e-12, err_msg=k)
        else:
            assert np.array_equal(m, p), (k, m, p)


@pytest.mark.parametrize("per", [(False, False, False), (True, True, False), (True, False, True)])
def test_marshal3d_matches_python_binding(gw, per):
    sim = cases.box3d_sim(per=per, axis=3 if not per[2] else 1)
    mex, _ = gw.call("marshal3d", sim)
    _same3d(mex, _py3d(sim))


def test_marshal3d_defaults_and_scalar_planes(gw):
    n = (20, 16, 24)
    d = 0.04
    x, y, z = (np.arange(m) * d for m in n)
    sim = dict(x=x, y=y, z=z, eps={c: np.full(n, 2.0) for c in "xyz"}, npml=6, periodic=np.array([True, True, False]),
               source=dict(axis=3, index=8, Ea=1.0, Hb=1.46, lambda0=0.6), lambdas=[0.6],
               monitors=[dict(axis=3, index=12)])
    mex, _ = gw.call("marshal3d", sim)
    _same3d(mex, _py3d(sim))
    assert list(np.ravel(mex["npml"])) == [0, 0, 6] and list(np.ravel(mex["periodic"])) == [1, 1, 0]
    assert mex["courant"] == 0.99 / math.sqrt(3) and mex["src_bw"] == 0.2 and mex["src_neff"] == 1.0
    np.testing.assert_allclose(np.ravel(mex["src_sums"]), [20 * 16 * 1.0, 0.0, 0.0, 20 * 16 * 1.46], rtol=1e-12)


@pytest.mark.parametrize("edit,ident", [
    (lambda s: s.pop("eps"), "orf:invalidInput"),
    (lambda s: s.update(pol="XY"), "orf:invalidInput"),
    (lambda s: s.update(x=np.r_[s["x"][:-1], s["x"][-1] + 0.005]), "orf:invalidInput"),
    (lambda s: s.update(eps=s["eps"][:, :-1]), "orf:invalidInput"),
    (lambda s: s.update(lambdas=[]), "orf:invalidInput"),
    (lambda s: s["source"].update(ix=3), "orf:invalidInput"),          # inside the CPML: the library's check
    (lambda s: s.update(monitors=[0]), "orf:invalidInput"),            # 1-based: 0 is outside the grid
    (lambda s: s.update(courant=0.9), "orf:invalidInput"),             # above the 2D Yee limit
    (lambda s: s.update(precision="half"), "orf:invalidInput"),
])
def test_malformed_sims_raise_invalid_input(gw, edit, ident):
    sim = cases.mixed_te_sim(seed=1)
    sim["source"] = dict(sim["source"])
    edit(sim)
    with pytest.raises(mexshim.MexError) as ei:
        gw.call("fdtd2D", sim)
    assert ei.value.identifier == ident, ei.value


def test_tm_needs_its_eps_components_and_te_wrapper_forces_te(gw):
    sim = cases.mixed_te_sim(seed=1, pol="TM")
    with pytest.raises(mexshim.MexError) as ei:
        gw.call("fdtd2DTE", sim)            # TE needs sim.eps, which a TM sim lacks
    assert ei.value.identifier == "orf:invalidInput" and "sim.eps" in ei.value.message
    bad = dict(sim, epsZ=sim["epsZ"][:-1])
    with pytest.raises(mexshim.MexError) as ei:
        gw.call("fdtd2D", bad)
    assert ei.value.identifier == "orf:invalidInput" and "epsZ" in ei.value.message


def test_usage_errors(gw):
    for args in [("nonsense", {"x": 1}), ("fdtd2D", [1, 2, 3])]:
        with pytest.raises(mexshim.MexError) as ei:
            gw.call(*args)
        assert ei.value.identifier == "orf:invalidInput"


def test_valid_run_without_a_device_raises_no_device(gw):
    if orf.device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(mexshim.MexError) as ei:
        gw.call("fdtd2D", cases.mixed_te_sim(seed=1))
    assert ei.value.identifier == "orf:noDevice"


# ------------------------------------------------------------ on the GPU ---
def _py_run2d(sim):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return orf.fdtd2D(sim)


@pytest.mark.gpu
@pytest.mark.parametrize("pol", ["TE", "TM"])
def test_gateway_run2d_equals_python_binding(gw, pol):
    sim = cases.mixed_te_sim(seed=6, pol=pol, steps=300)
    out, w = gw.call("fdtd2D", sim)
    ref = _py_run2d(sim)
    assert w == "fdtd2D:notConverged"        # shutoff 0: the run ends at maxTime
    for k in ("flux", "fluxZ", "P", "B", "PZ", "AZ"):
        assert np.array_equal(np.reshape(out[k], ref[k].shape), ref[k]), k
    alias = {"TE": dict(Ey="P", Hz="B", EyZ="PZ", HxZ="AZ"), "TM": dict(Hy="P", Ez="B", HyZ="PZ", ExZ="AZ")}[pol]
    for k, base in alias.items():
        sign = -1 if k in ("Ez", "ExZ") else 1
        assert np.array_equal(np.reshape(out[k], ref[base].shape), sign * ref[base]), k
    assert out["steps"] == ref["steps"] == 300 and out["converged"] is False
    assert out["time"] == ref["time"]


@pytest.mark.gpu
def test_gateway_progress_error_is_rethrown_unchanged(gw):
    sim = cases.mixed_te_sim(seed=7, steps=2000)
    calls = []

    def progress(frac, msg):
        calls.append(frac)
        return len(calls) >= 2      # the second call throws (orf:cancelled)

    with pytest.raises(mexshim.MexError) as ei:
        gw.call("fdtd2D", dict(sim, progress=progress))
    assert ei.value.identifier == "orf:cancelled"
    assert len(calls) == 2


@pytest.mark.gpu
def test_gateway_run3d_equals_python_binding(gw):
    sim = cases.box3d_sim(steps=120, seed=2)
    out, w = gw.call("fdtd3D", sim)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        ref = orf.fdtd3D(sim)
    assert w == "fdtd3D:notConverged"
    assert np.array_equal(np.reshape(out["flux"], ref["flux"].shape), ref["flux"])
    mons = out["mon"] if isinstance(out["mon"], list) else [out["mon"]]
    for mo, mr in zip(mons, ref["mon"]):
        for k in ("Ea", "Eb", "Ha", "Hb"):
            assert np.array_equal(np.reshape(mo[k], mr[k].shape), mr[k]), k
    assert out["steps"] == ref["steps"]


# ------------------------------------------------- the FDFD commands ------
def _fdfd_args(nx=40, nz=30, seed=3):
    from tests import fdfd_cases
    x, z, eps, lam, J, g, npml = fdfd_cases.random_problem(nx, nz, seed)
    return x, z, eps, lam, J, g, npml


@pytest.mark.parametrize("edit,frag", [
    (lambda a: a.__setitem__(0, np.array([0.0, 0.1, 0.3, 0.4])), "uniform"),
    (lambda a: a.__setitem__(1, a[1] * 2.0), "same spacing"),
    (lambda a: a.__setitem__(2, a[2][:, :-1]), "nx x nz"),
    (lambda a: a.__setitem__(4, np.array([1.0, 2.0, 3.0])), "Npml"),
])
def test_fdfd_factor_rejects_malformed_input(gw, edit, frag):
    x, z, eps, lam, J, g, npml = _fdfd_args()
    a = [x, z, eps, lam, np.asarray(npml, dtype=float), 1e-8]
    edit(a)
    with pytest.raises(mexshim.MexError) as ei:
        gw.call_args("fdfd2D_factor", *a)
    assert ei.value.identifier == "orf:invalidInput" and frag in ei.value.message


def test_fdfd_commands_reject_usage_and_unknown_ids(gw):
    with pytest.raises(mexshim.MexError) as ei:
        gw.call_args("fdfd2D_factor", np.arange(5.0))
    assert ei.value.identifier == "orf:invalidInput"
    for args in [("fdfd2D_solve", 7.0, np.zeros((3, 3)), 0.0), ("fdfd2D_release", 65.0), ("fdfd2D_release", 1.5)]:
        with pytest.raises(mexshim.MexError) as ei:
            gw.call_args(*args)
        assert ei.value.identifier == "orf:invalidInput"


def test_fdfd_factor_without_a_device_raises_no_device(gw):
    if orf.device_count() > 0:
        pytest.skip("a GPU is present")
    x, z, eps, lam, J, g, npml = _fdfd_args()
    with pytest.raises(mexshim.MexError) as ei:
        gw.call_args("fdfd2D_factor", x, z, eps, lam, np.asarray(npml, dtype=float), 1e-8)
    assert ei.value.identifier == "orf:noDevice"


@pytest.mark.gpu
def test_gateway_fdfd_equals_python_binding(gw):
    x, z, eps, lam, J, g, npml = _fdfd_args(60, 44, 5)
    fid = gw.call_args("fdfd2D_factor", x, z, eps, lam, np.asarray(npml, dtype=float), 1e-8)
    E = gw.call_args("fdfd2D_solve", fid, np.real(J), 0.0)      # a real current is accepted
    lam_ = gw.call_args("fdfd2D_solve", fid, g.ravel(order="F"), 1.0)
    o = orf.fdfd2D(x, z, eps, lam, np.real(J), Npml=npml)
    assert np.array_equal(np.reshape(E, o.E.shape), o.E)
    assert np.array_equal(np.reshape(lam_, o.E.shape), o.adjoint(g))
    o.close()
    assert gw.call_args("fdfd2D_release", fid) is None
    with pytest.raises(mexshim.MexError) as ei:
        gw.call_args("fdfd2D_solve", fid, np.real(J), 0.0)
    assert ei.value.identifier == "orf:invalidInput"
