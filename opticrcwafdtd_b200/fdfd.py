"""orf.fdfd2D: the 2D TE frequency-domain solver with its adjoint
(toolbox/+orf/fdfd2D.m:1-19), factored and solved on the device through
orf_fdfd2d_* in include/orf_fdtd.h.

    out = fdfd2D(x, z, epsr, lambda0, J, Npml=(30, 30), PmlReflection=1e-8)

solves (1/s_x) d/dx((1/s_x) dE/dx) + (1/s_z) d/dz((1/s_z) dE/dz) + k0^2 eps E
= -J for E = E_y on the grid's points (those of orf.fdtd2DTE) with E = 0
outside and stretched-coordinate PML.  The result keeps the device factors:
out.solve(J2) solves for another current, out.adjoint(g) solves A.' lam = g
(for c = sum(g .* E), dc/deps = -k0^2 lam .* E, fdfd2D.m:13-15), and
out.fluxX(ix, iz) / out.fluxZ(iz, ix) give the power through a vertical /
horizontal line from centred differences of E (fdfd2D.m:16-18; 1-based
indices as in the reference's calls, > 0 toward +x / +z).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi, _lib


def _axis(v, name):
    v = np.asarray(v, dtype=np.float64).ravel()
    if v.size < 3:
        raise _abi.OrfError("orf:invalidInput", f"{name} needs at least three points")
    d = float(v[1] - v[0])
    if not (d > 0) or np.max(np.abs(np.diff(v) - d)) > 1e-9 * max(1.0, abs(d)) * v.size:
        raise _abi.OrfError("orf:invalidInput", f"{name} must be uniform and increasing")
    return v, d


def _cfield(a, nx, nz, name):
    a = np.asarray(a)
    if a.size != nx * nz:
        raise _abi.OrfError("orf:invalidInput", f"{name} must be {nx} x {nz}, got {a.shape}")
    # nx x nz, or its column-major vector (MATLAB's A(:))
    a = a.reshape((nx, nz), order="F")
    return np.asfortranarray(a.astype(np.complex128))


class FDFD2D:
    """Factored 2D TE operator on the device; see the module docstring."""

    def __init__(self, x, z, epsr, lambda0, J, Npml=(30, 30), PmlReflection=1e-8, ctx=None):
        from .fdtd import Context
        self.handle = None
        self.lib = _lib.load()
        x, dx = _axis(x, "x")
        z, dz = _axis(z, "z")
        if abs(dx - dz) > 1e-9 * dx:
            raise _abi.OrfError("orf:invalidInput", "x and z must have the same spacing")
        self.x, self.z, self.d = x, z, dx
        self.nx, self.nz = x.size, z.size
        self.k0 = 2.0 * np.pi / float(lambda0)
        npml = np.atleast_1d(np.asarray(Npml, dtype=np.int64)).ravel()
        if npml.size == 1:
            npml = np.repeat(npml, 2)
        eps = _cfield(epsr, self.nx, self.nz, "epsr")
        self._own_ctx = ctx is None
        self.ctx = Context(0) if ctx is None else ctx
        flat = eps.ravel(order="F")
        pr = _abi.OrfFdfd2D(self.nx, self.nz, dx, flat.view(np.float64).ctypes.data_as(_abi.c_double_p),
                            float(lambda0), int(npml[0]), int(npml[1]), float(PmlReflection))
        h = C.c_void_p()
        _lib.check(self.lib.orf_fdfd2d_factor(self.ctx.handle, C.byref(pr), C.byref(h)), "fdfd2D")
        self.handle = h
        self.E = self.solve(J)

    def info(self) -> dict:
        m, nb, cl = C.c_int32(), C.c_int32(), C.c_int32()
        _lib.check(self.lib.orf_fdfd2d_info(self.handle, C.byref(m), C.byref(nb), C.byref(cl)), "fdfd2D info")
        return {"block": m.value, "blocks": nb.value, "cluster": cl.value}

    def _run(self, v, transpose: int) -> np.ndarray:
        if self.handle is None:
            raise _abi.OrfError("orf:invalidInput", "fdfd2D: the factors were released")
        rhs = _cfield(v, self.nx, self.nz, "right-hand side").ravel(order="F")
        out = np.empty(self.nx * self.nz, dtype=np.complex128)
        _lib.check(self.lib.orf_fdfd2d_solve(self.handle, rhs.view(np.float64).ctypes.data_as(_abi.c_double_p),
                                             out.view(np.float64).ctypes.data_as(_abi.c_double_p), transpose),
                   "fdfd2D solve")
        return out.reshape((self.nx, self.nz), order="F")

    def solve(self, J2) -> np.ndarray:
        """E for another current J2 with the same factors (A E = -J2)."""
        return self._run(J2, 0)

    def adjoint(self, g) -> np.ndarray:
        """lam with A.' lam = g (g: nx x nz or its column-major vector)."""
        return self._run(g, 1)

    def fluxX(self, ix, iz) -> float:
        """Power through the vertical line x(ix) over the z indices iz (1-based)."""
        i = int(ix) - 1
        k = np.asarray(iz, dtype=np.int64).ravel() - 1
        E = self.E
        dE = (E[i + 1, k] - E[i - 1, k]) / (2.0 * self.d)
        return float(self.d / (2.0 * self.k0) * np.sum(np.imag(np.conj(E[i, k]) * dE)))

    def fluxZ(self, iz, ix) -> float:
        """Power through the horizontal line z(iz) over the x indices ix (1-based)."""
        k = int(iz) - 1
        i = np.asarray(ix, dtype=np.int64).ravel() - 1
        E = self.E
        dE = (E[i, k + 1] - E[i, k - 1]) / (2.0 * self.d)
        return float(self.d / (2.0 * self.k0) * np.sum(np.imag(np.conj(E[i, k]) * dE)))

    def close(self) -> None:
        if getattr(self, "handle", None) is not None:
            self.lib.orf_fdfd2d_release(self.handle)
            self.handle = None
        if getattr(self, "_own_ctx", False) and getattr(self, "ctx", None) is not None:
            self.ctx.close()
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fdfd2D(x, z, epsr, lambda0, J, Npml=(30, 30), PmlReflection=1e-8, ctx=None) -> FDFD2D:
    """out = orf.fdfd2D(x, z, epsr, lambda0, J) (toolbox/+orf/fdfd2D.m:1-19)."""
    return FDFD2D(x, z, epsr, lambda0, J, Npml=Npml, PmlReflection=PmlReflection, ctx=ctx)
