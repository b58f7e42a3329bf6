"""ctypes front end of the C++ oracle (oracle/fdtd_oracle.cpp).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).  Mirrors orf.fdtd2D /
orf.fdtd2DTE / orf.fdtd3D (toolbox/+orf/fdtd2D.m:1-29, fdtd2DTE.m:33-34,
fdtd3D.m:1-29) on the CPU, in FP64 (precision "double") or with FP32 fields
(precision "single"; DFT sums stay FP64 as in fdtd2DTE.m:24-25).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import warnings

import numpy as np

from opticrcwafdtd_b200 import _abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "liborf_oracle.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        lib = C.CDLL(_SO)
        dpp = C.POINTER(C.POINTER(C.c_double))
        lib.oracle_fdtd2d_run.argtypes = [C.POINTER(_abi.OrfSim2D), C.POINTER(_abi.OrfOut2D),
                                          _abi.PROGRESS_FN, C.c_void_p, C.c_int, dpp]
        lib.oracle_fdtd3d_run.argtypes = [C.POINTER(_abi.OrfSim3D), C.POINTER(_abi.OrfOut3D),
                                          _abi.PROGRESS_FN, C.c_void_p, C.c_int, dpp]
        lib.oracle_pulse.restype = C.c_double
        lib.oracle_pulse.argtypes = [C.c_double, C.c_double, C.c_double]
        lib.oracle_max_threads.restype = C.c_int
        _lib = lib
    return _lib


def max_threads() -> int:
    return int(load().oracle_max_threads())


def pulse(lambda0: float, bw: float, t: float) -> float:
    return float(load().oracle_pulse(lambda0, bw, t))


def _check(st: int, box, name: str):
    if box and "exc" in box:
        raise box["exc"]
    if st != 0:
        raise _abi.OrfError(_abi.STATUS_IDS.get(st, "orf:error"), f"oracle {name} failed", st)


def _field_ptrs(shapes):
    arrs = [np.zeros(s, order="F") for s in shapes]
    ptrs = (C.POINTER(C.c_double) * len(arrs))(*[a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs])
    return arrs, ptrs


def fdtd2D(sim, threads: int = 0, fields: bool = False) -> dict:
    """Oracle orf.fdtd2D; with fields=True out['fields'] = [P, A, B] at the end."""
    m = _abi.marshal_sim2d(sim)
    o, bufs = _abi.alloc_out2d(m)
    cb, box = _abi.make_progress(_abi._get(sim, "progress"))
    arrs, ptrs = None, None
    if fields:
        nx, nz = m.meta["nx"], m.meta["nz"]
        per = bool(m.struct.periodic_z)
        arrs, ptrs = _field_ptrs([(nx, nz), (nx, nz if per else nz - 1), (nx - 1, nz)])
    st = load().oracle_fdtd2d_run(C.byref(m.struct), C.byref(o), cb or _abi.PROGRESS_FN(0), None, threads, ptrs)
    _check(st, box, "fdtd2D")
    out = _abi.finish_out2d(m, o, bufs)
    if fields:
        out["fields"] = arrs
    if not out["converged"]:
        warnings.warn("fdtd2D:notConverged: maxTime reached before the shutoff", _abi.NotConvergedWarning)
    return out


def fdtd2DTE(sim, threads: int = 0, fields: bool = False) -> dict:
    sim = dict(sim)
    sim["pol"] = "TE"
    return fdtd2D(sim, threads, fields)


def fdtd3D(sim, threads: int = 0, fields: bool = False) -> dict:
    """Oracle orf.fdtd3D; with fields=True out['fields'] = [Ex Ey Ez Hx Hy Hz]."""
    m = _abi.marshal_sim3d(sim)
    o, bufs = _abi.alloc_out3d(m)
    cb, box = _abi.make_progress(_abi._get(sim, "progress"))
    arrs, ptrs = None, None
    if fields:
        arrs, ptrs = _field_ptrs([tuple(m.meta["n"])] * 6)
    st = load().oracle_fdtd3d_run(C.byref(m.struct), C.byref(o), cb or _abi.PROGRESS_FN(0), None, threads, ptrs)
    _check(st, box, "fdtd3D")
    out = _abi.finish_out3d(m, o, bufs)
    if fields:
        out["fields"] = arrs
    if not out["converged"]:
        warnings.warn("fdtd3D:notConverged: maxTime reached before the shutoff", _abi.NotConvergedWarning)
    return out
