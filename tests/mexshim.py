"""Python side of the MEX-gateway tests: compiles opticrcwafdtd_b200/matlab/
orf_fdtd_mex.c against the project-written mex.h / matrix.h stand-in in
tests/mex_shim (no MATLAB here), converts MATLAB-style values between Python
and the stand-in's mxArrays, and calls the gateway the way MATLAB would.
Test infrastructure only."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "tests", "mex_shim")
GATEWAY = os.path.join(ROOT, "opticrcwafdtd_b200", "matlab", "orf_fdtd_mex.c")
LIBDIR = os.path.join(ROOT, "opticrcwafdtd_b200", "lib")

CLS_STRUCT, CLS_LOGICAL, CLS_CHAR, CLS_DOUBLE, CLS_FUNCTION, CLS_OBJECT = 1, 2, 3, 4, 5, 6
CALLBACK = C.CFUNCTYPE(C.c_int, C.c_double, C.c_char_p)


class MexError(Exception):
    def __init__(self, identifier, message):
        super().__init__(f"{identifier}: {message}")
        self.identifier = identifier
        self.message = message


def build(outdir: str) -> str:
    """Compile gateway + stand-in into one shared library, linked to liborf_fdtd.so."""
    so = os.path.join(outdir, "orf_fdtd_mex_shim.so")
    cmd = ["gcc", "-std=c11", "-O1", "-Wall", "-Wextra", "-Werror", "-Wno-unused-parameter", "-fPIC", "-shared",
           "-I", SHIM, "-I", os.path.join(ROOT, "include"), GATEWAY, os.path.join(SHIM, "mexshim.c"),
           "-L", LIBDIR, "-lorf_fdtd", f"-Wl,-rpath,{LIBDIR}", "-lm", "-o", so]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return so


class Gateway:
    def __init__(self, so: str):
        L = C.CDLL(so)
        vp = C.c_void_p
        sz = C.c_size_t
        sigs = {
            "shim_double": (vp, [sz, C.POINTER(sz), C.c_void_p, C.c_int]),
            "shim_logical": (vp, [C.c_int]), "shim_logicals": (vp, [sz, C.c_char_p]),
            "shim_string": (vp, [C.c_char_p]), "shim_struct": (vp, [sz]),
            "shim_set": (None, [vp, sz, C.c_char_p, vp]), "shim_handle": (vp, [CALLBACK]),
            "shim_call": (C.c_int, [C.c_int, C.POINTER(vp), C.c_int, C.POINTER(vp)]),
            "shim_error_id": (C.c_char_p, []), "shim_error_msg": (C.c_char_p, []),
            "shim_warning_id": (C.c_char_p, []), "shim_get": (vp, [vp, sz, C.c_char_p]),
            "shim_nfields": (C.c_int, [vp]), "shim_field_name": (C.c_char_p, [vp, C.c_int]),
            "shim_class": (C.c_int, [vp]), "shim_is_complex": (C.c_int, [vp]), "shim_numel": (sz, [vp]),
            "shim_ndims": (sz, [vp]), "shim_dim": (sz, [vp, sz]), "shim_data": (vp, [vp]),
            "shim_free": (None, [vp]),
        }
        for n, (r, a) in sigs.items():
            f = getattr(L, n)
            f.restype = r
            f.argtypes = a
        self.L = L
        self._keep = []

    # ---- Python -> mxArray
    def to_mx(self, v):
        L = self.L
        if isinstance(v, str):
            return L.shim_string(v.encode())
        if callable(v):
            cb = CALLBACK(lambda frac, msg: int(bool(v(frac, msg.decode() if msg else ""))))
            self._keep.append(cb)
            return L.shim_handle(cb)
        if isinstance(v, dict):
            s = L.shim_struct(1)
            for k, x in v.items():
                L.shim_set(s, 0, k.encode(), self.to_mx(x))
            return s
        if isinstance(v, (list, tuple)) and v and all(isinstance(e, dict) for e in v):
            s = L.shim_struct(len(v))
            for i, e in enumerate(v):
                for k, x in e.items():
                    L.shim_set(s, i, k.encode(), self.to_mx(x))
            return s
        a = np.asarray(v)
        if a.dtype == bool:
            if a.ndim == 0:
                return L.shim_logical(int(a))
            b = np.ascontiguousarray(a.ravel(order="F"), dtype=np.uint8)
            return L.shim_logicals(b.size, b.tobytes())
        cplx = np.iscomplexobj(a)
        a = np.asfortranarray(a, dtype=np.complex128 if cplx else np.float64)
        dims = a.shape if a.ndim >= 2 else ((1, a.size) if a.ndim == 1 else (1, 1))
        d = (C.c_size_t * len(dims))(*dims)
        return L.shim_double(len(dims), d, a.ctypes.data_as(C.c_void_p), 1 if cplx else 0)

    # ---- mxArray -> Python
    def from_mx(self, p):
        L = self.L
        cls = L.shim_class(p)
        if cls == CLS_STRUCT:
            n = L.shim_numel(p)
            names = [L.shim_field_name(p, f).decode() for f in range(L.shim_nfields(p))]
            recs = [{k: self.from_mx(L.shim_get(p, i, k.encode())) for k in names} for i in range(n)]
            return recs[0] if n == 1 else recs
        if cls == CLS_LOGICAL:
            return bool(C.cast(L.shim_data(p), C.POINTER(C.c_bool))[0])
        dims = tuple(L.shim_dim(p, k) for k in range(L.shim_ndims(p)))
        n = L.shim_numel(p)
        cplx = L.shim_is_complex(p)
        if n == 0:
            return np.zeros(dims, dtype=np.complex128 if cplx else np.float64)
        buf = (C.c_double * (n * (2 if cplx else 1))).from_address(L.shim_data(p))
        a = np.frombuffer(buf, dtype=np.float64).copy()
        if cplx:
            a = a.view(np.complex128)
        a = a.reshape(dims, order="F")
        return a.item() if a.size == 1 and dims == (1, 1) else a

    def call_args(self, cmd: str, *args):
        """out = orf_fdtd_mex(cmd, args...); raises MexError; returns the
        output (None when the command returns nothing)."""
        mx = [self.to_mx(cmd)] + [self.to_mx(a) for a in args]
        prhs = (C.c_void_p * len(mx))(*mx)
        plhs = (C.c_void_p * 1)()
        if self.L.shim_call(1, plhs, len(mx), prhs):
            raise MexError(self.L.shim_error_id().decode(), self.L.shim_error_msg().decode())
        return self.from_mx(plhs[0]) if plhs[0] else None

    def call(self, cmd: str, sim=None):
        """out = orf_fdtd_mex(cmd, sim); raises MexError with MATLAB's
        identifier; returns (out, warning identifier or None)."""
        args = [self.to_mx(cmd)] + ([self.to_mx(sim)] if sim is not None else [])
        prhs = (C.c_void_p * len(args))(*args)
        plhs = (C.c_void_p * 1)()
        if self.L.shim_call(1, plhs, len(args), prhs):
            raise MexError(self.L.shim_error_id().decode(), self.L.shim_error_msg().decode())
        w = self.L.shim_warning_id().decode() or None
        return self.from_mx(plhs[0]), w
