"""CPU oracle of the 2D TE frequency-domain solver -- TEST INFRASTRUCTURE ONLY.

Restates the problem toolbox/+orf/fdfd2D.m:1-19 documents (the solver itself
is distributed as P-code, toolbox/+orf/fdfd2D.p, and cannot run here):

    (1/s_x) d/dx((1/s_x) dE/dx) + (1/s_z) d/dz((1/s_z) dE/dz) + k0^2 eps E = -J

for E = E_y on the FDTD's E_y points (fdtd2DTE.m:8), E = 0 outside the
grid, stretched-coordinate PML s = 1 + i a (delta/L)^3 with the e^{-i w t}
convention (outgoing waves decay), `Npml` cells per side (default 30 x 30)
and a normal-incidence reflection `PmlReflection` (default 1e-8).  The
adjoint solves A.' lam = g with the same matrix (fdfd2D.m:13-15), so that a
figure of merit c = sum(g .* E) has dc/deps = -k0^2 lam .* E.  The fluxes
(fdfd2D.m:16-18) are (d / (2 k0)) sum Im(conj(E) dE/dn) over the line with
centred differences, > 0 toward +x / +z.

Discretisation choices the reference does not document (the engine makes
the same ones): the layer depth at position u (integer points u = i, half
points u = i + 1/2, 0-based) is npml - u below the low edge npml and
u - (n - 1 - npml) above the high edge, as the FDTD's CPML profile; the
strength a = 2 ln(1/R) / (k0 L), L = npml d, so that a normal plane wave
crossing the layer twice is attenuated by R in the continuum.  Parity is
pinned on the reference's own physics checks for this solver
(tests/TestInverseDesign.m:12-33: lossless guide 1e-5, even split 1e-4,
the Yee-dispersion phase velocity 1e-5) and on an adjoint gradient against
finite differences; bit parity with the P-code is unpinned.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def stretch(n: int, npml: int, d: float, k0: float, R: float, half: bool) -> np.ndarray:
    """s at the n integer points (half=False) or the n+1 half points
    u = -1/2 .. n-1/2 (half=True) of one axis."""
    u = np.arange(n + 1) - 0.5 if half else np.arange(n, dtype=np.float64)
    s = np.ones(u.size, dtype=np.complex128)
    if npml <= 0:
        return s
    L = npml * d
    a = 2.0 * np.log(1.0 / R) / (k0 * L)
    lo, hi = float(npml), float(n - 1 - npml)
    depth = np.where(u < lo, lo - u, np.where(u > hi, u - hi, 0.0)) * d
    return 1.0 + 1j * a * (depth / L) ** 3


def operator(nx: int, nz: int, d: float, eps: np.ndarray, k0: float, npml=(30, 30), R: float = 1e-8):
    """The sparse matrix A of A E = -J, unknown (i, k) at i + nx k (MATLAB
    column-major order of an nx x nz array)."""
    sxi = stretch(nx, npml[0], d, k0, R, False)
    sxh = stretch(nx, npml[0], d, k0, R, True)     # sxh[i] at u = i - 1/2
    szi = stretch(nz, npml[1], d, k0, R, False)
    szh = stretch(nz, npml[1], d, k0, R, True)
    I = np.arange(nx)[:, None] * np.ones((1, nz), dtype=np.int64)
    K = np.ones((nx, 1), dtype=np.int64) * np.arange(nz)[None, :]
    idx = I + nx * K
    h2 = 1.0 / (d * d)
    cxm = h2 / (sxi[I] * sxh[I])          # to (i-1, k)
    cxp = h2 / (sxi[I] * sxh[I + 1])      # to (i+1, k)
    czm = h2 / (szi[K] * szh[K])
    czp = h2 / (szi[K] * szh[K + 1])
    diag = -(cxm + cxp + czm + czp) + k0 * k0 * np.asarray(eps, dtype=np.complex128)
    rows = [idx.ravel("F")]
    cols = [idx.ravel("F")]
    vals = [diag.ravel("F")]
    for m, c, di, dk in ((I > 0, cxm, -1, 0), (I < nx - 1, cxp, 1, 0), (K > 0, czm, 0, -1), (K < nz - 1, czp, 0, 1)):
        rows.append(idx[m])
        cols.append((I + di + nx * (K + dk))[m])
        vals.append(c[m])
    N = nx * nz
    return sp.csc_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))


class FDFD2D:
    """orf.fdfd2D(x, z, epsr, lambda0, J) on the CPU: E, k0, solve(J2),
    adjoint(g), fluxX(ix, iz), fluxZ(iz, ix) (indices 1-based, as in the
    reference's calls)."""

    def __init__(self, x, z, epsr, lambda0, J, Npml=(30, 30), PmlReflection=1e-8):
        x = np.asarray(x, dtype=np.float64).ravel()
        z = np.asarray(z, dtype=np.float64).ravel()
        self.nx, self.nz = x.size, z.size
        self.d = float(x[1] - x[0])
        self.k0 = 2.0 * np.pi / float(lambda0)
        self.A = operator(self.nx, self.nz, self.d, np.asarray(epsr), self.k0, tuple(int(v) for v in Npml),
                          float(PmlReflection))
        self.lu = spla.splu(self.A)
        self.E = self.solve(J)

    def solve(self, J):
        b = -np.asarray(J, dtype=np.complex128).reshape((self.nx, self.nz), order="F").ravel("F")
        return self.lu.solve(b).reshape((self.nx, self.nz), order="F")

    def adjoint(self, g):
        b = np.asarray(g, dtype=np.complex128).reshape((self.nx, self.nz), order="F").ravel("F")
        return self.lu.solve(b, trans="T").reshape((self.nx, self.nz), order="F")

    def fluxX(self, ix, iz):
        i = int(ix) - 1
        k = np.asarray(iz, dtype=np.int64).ravel() - 1
        E = self.E
        dE = (E[i + 1, k] - E[i - 1, k]) / (2 * self.d)
        return float(self.d / (2 * self.k0) * np.sum(np.imag(np.conj(E[i, k]) * dE)))

    def fluxZ(self, iz, ix):
        k = int(iz) - 1
        i = np.asarray(ix, dtype=np.int64).ravel() - 1
        E = self.E
        dE = (E[i, k + 1] - E[i, k - 1]) / (2 * self.d)
        return float(self.d / (2 * self.k0) * np.sum(np.imag(np.conj(E[i, k]) * dE)))


def fdfd2D(x, z, epsr, lambda0, J, **opts) -> FDFD2D:
    return FDFD2D(x, z, epsr, lambda0, J, **opts)
