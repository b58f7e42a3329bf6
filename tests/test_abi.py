"""The C ABI library: loads without a GPU, exports exactly what include/orf_fdtd.h
declares, and rejects malformed sims on the host (no device needed)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from opticrcwafdtd_b200 import _abi, _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "orf_fdtd.h")).read()
    return sorted(set(re.findall(r"^ORF_API\s+[\w\s\*]+?\b(orf_\w+)\(", src, re.M)))


def test_library_exports_every_header_symbol():
    lib = _lib.load()
    names = header_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.exported_names())
    assert lib.orf_abi_version() == 1


def _sim(**kw):
    s = dict(x=np.arange(40) * 0.02, z=np.arange(20) * 0.02, eps=np.ones((40, 20)), npml=[5, 5],
             source=dict(ix=10, profile=np.ones(20), neff=1, lambda0=1.5), lambdas=[1.5], monitors=[8, 30])
    s.update(kw)
    return s


@pytest.mark.parametrize("bad,frag", [
    (dict(source=dict(ix=3, profile=np.ones(20), neff=1, lambda0=1.5)), "inside the CPML"),
    (dict(monitors=[0]), "outside"),
    (dict(monitors=[41]), "outside"),
    (dict(eps=-np.ones((40, 20))), "positive"),
    (dict(courant=0.9), "stability"),
    (dict(npml=[25, 5]), "does not fit"),
    (dict(lambdas=[-1.0]), "positive"),
])
def test_host_validation_rejects_bad_sims(bad, frag):
    lib = _lib.load()
    m = _abi.marshal_sim2d(_sim(**bad))
    o, _ = _abi.alloc_out2d(m)
    st = lib.orf_fdtd2d_run(C.byref(m.struct), C.byref(o), _abi.PROGRESS_FN(0), None)
    assert st == 1, _lib.last_error()
    assert frag in _lib.last_error()


def test_permittivity_scan_reports_the_first_bad_cell_of_long_arrays():
    """Arrays of millions of values are scanned by several host threads in
    blocks: the message names the first bad cell in column-major order, even
    when later blocks (scanned by other threads) fail too."""
    lib = _lib.load()
    nx, nz = 2000, 1100
    for bad_at, vals in (((1_650_000, 700_001, 2_100_000), (np.nan, -2.0, np.inf)),
                         ((4095, 4096), (0.0, np.nan)),
                         ((nx * nz - 1,), (np.inf,))):
        eps = np.ones((nx, nz), order="F")
        flat = eps.reshape(-1, order="F")   # a view: column-major cell order
        for q, v in zip(bad_at, vals):
            flat[q] = v
        s = dict(x=np.arange(nx) * 0.02, z=np.arange(nz) * 0.02, eps=eps, npml=[5, 5],
                 source=dict(ix=10, profile=np.ones(nz), neff=1, lambda0=1.5), lambdas=[1.5], monitors=[8])
        m = _abi.marshal_sim2d(s)
        o, _ = _abi.alloc_out2d(m)
        st = lib.orf_fdtd2d_run(C.byref(m.struct), C.byref(o), _abi.PROGRESS_FN(0), None)
        assert st == 1
        first = min(bad_at)
        assert f"sim.eps({first + 1})" in _lib.last_error(), _lib.last_error()


def test_marshal_rejects_wrong_shapes():
    with pytest.raises(_abi.OrfError) as e:
        _abi.marshal_sim2d(_sim(eps=np.ones((39, 20))))
    assert e.value.identifier == "orf:invalidInput"
    with pytest.raises(_abi.OrfError):
        _abi.marshal_sim2d(_sim(pol="XX"))
    with pytest.raises(_abi.OrfError):
        _abi.marshal_sim2d(_sim(z=np.array([0, 0.02, 0.05])))


def test_no_device_fails_loudly_without_fallback():
    import opticrcwafdtd_b200 as orf
    if orf.device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(_abi.OrfError) as e:
        orf.fdtd2DTE(_sim())
    assert e.value.identifier == "orf:noDevice"
    # the GPU permittivity generator and 3D runs refuse as well: no host path
    x = (np.arange(8) + 0.5) * 0.02
    with pytest.raises(_abi.OrfError) as e:
        orf.epsComponents3D(x, x, x, 1.0, [["box", [0, 0.1, 0, 0.1, 0, 0.1, 2.0]]], device=True)
    assert e.value.identifier == "orf:noDevice"
    from tests import cases
    with pytest.raises(_abi.OrfError) as e:
        orf.fdtd3D(cases.box3d_sim(n=(20, 18, 24), steps=10))
    assert e.value.identifier == "orf:noDevice"


def _header_struct_fields(name):
    """Field names of `typedef struct name { ... } name;` in the header, in order."""
    src = open(os.path.join(ROOT, "include", "orf_fdtd.h")).read()
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), src, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        # "type a, b[3], *c" -> a, b, c
        for part in re.split(r",", decl):
            m = re.search(r"\**\s*(\w+)\s*(\[[^\]]*\])*\s*$", part.strip())
            names.append(m.group(1))
    return names


@pytest.mark.parametrize("cname,pyname", [
    ("orf_sim2d", "OrfSim2D"), ("orf_out2d", "OrfOut2D"), ("orf_sim3d", "OrfSim3D"), ("orf_out3d", "OrfOut3D"),
    ("orf_tuning", "OrfTuning"), ("orf_kernel_stats", "OrfKernelStats"), ("orf_serve_cfg", "OrfServeCfg"),
    ("orf_serve_job_info", "OrfServeJobInfo"), ("orf_eps_shape", "OrfEpsShape"),
])
def test_ctypes_mirrors_match_header_structs(cname, pyname):
    fields = [f[0] for f in getattr(_abi, pyname)._fields_]
    assert fields == _header_struct_fields(cname)


def _sim3d(**kw):
    from tests import cases
    s = cases.box3d_sim(n=(20, 18, 24), steps=10)
    s.update(kw)
    return s


@pytest.mark.parametrize("change,frag", [
    (lambda s: s["eps"].update(x=-np.ones_like(s["eps"]["x"])), "positive"),
    (lambda s: s.update(courant=0.6), "stability"),
    (lambda s: s.update(npml=[12, 5, 7]), "does not fit"),
    (lambda s: s["source"].update(index=2), "inside the CPML"),
    (lambda s: s.update(monitors=[dict(axis=3, index=25)]), "outside the grid"),
    (lambda s: s.update(lambdas=[0.6, -1.0]), "positive"),
])
def test_host_validation_rejects_bad_3d_sims(change, frag):
    """3D sims are validated on the host before any device work
    (fdtd3D.m:11-24 field rules), with the reference's messages."""
    lib = _lib.load()
    s = _sim3d()
    s["eps"] = dict(s["eps"])
    s["source"] = dict(s["source"])
    change(s)
    m = _abi.marshal_sim3d(s)
    o, _ = _abi.alloc_out3d(m)
    st = lib.orf_fdtd3d_run(C.byref(m.struct), C.byref(o), _abi.PROGRESS_FN(0), None)
    assert st == 1, _lib.last_error()
    assert frag in _lib.last_error()


def test_3d_permittivity_scan_reports_the_first_bad_cell():
    """The 3D scan (three components of over a million cells each, threaded
    in blocks) names the component and the first bad cell of it."""
    lib = _lib.load()
    s = _sim3d()
    n = (110, 100, 96)
    d = 0.04
    s.update(x=np.arange(n[0]) * d, y=np.arange(n[1]) * d, z=np.arange(n[2]) * d)
    s["eps"] = {c: np.ones(n, order="F") for c in "xyz"}
    s["source"] = dict(s["source"], Ea=1.0, Eb=0.0, Ha=0.0, Hb=1.0, index=20)
    s["monitors"] = [dict(axis=3, index=30)]
    flat = s["eps"]["y"].reshape(-1, order="F")
    flat[900_001] = np.nan
    flat[300_000] = -1.0
    m = _abi.marshal_sim3d(s)
    o, _ = _abi.alloc_out3d(m)
    st = lib.orf_fdtd3d_run(C.byref(m.struct), C.byref(o), _abi.PROGRESS_FN(0), None)
    assert st == 1
    assert "sim.eps.y(300001)" in _lib.last_error(), _lib.last_error()
