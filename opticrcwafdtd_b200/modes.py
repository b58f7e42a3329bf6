"""Slab-mode source profiles (host-side preparation of sim.source).

Restates toolbox/+orf/slabModes.m:1-57 (open code in the reference): guided
modes of a 1D index profile n(z) by second-order finite differences with
Dirichlet walls, on the FDTD's own z grid so the mode matches the Yee
discretisation.  The matrix is tridiagonal (slabModes.m:29-43); its leading
eigenpairs come from scipy's tridiagonal solver after a diagonal similarity
transform makes the TM matrix symmetric, instead of a dense eig of the full
matrix.  Eigenvalues are identical to rounding.
"""
from __future__ import annotations

import numpy as np
from scipy.linalg import eigh_tridiagonal


def slabModes(z, n, lambda0: float, pol: str = "TE", nModes: int = 1, EpsHalf=None) -> dict:
    """modes = slabModes(z, n, lambda0, pol, nModes, EpsHalf=...).

    Returns {"neff": (nModes,), "field": (numel(z), nModes)}, neff descending,
    each field scaled so max |field| = 1 with a positive peak (slabModes.m:44-52).
    """
    z = np.asarray(z, dtype=float).ravel()
    n = np.asarray(n).ravel()
    if n.size != z.size:
        raise ValueError("slabModes:size: n must match z.")
    pol = str(pol).upper()
    dz = z[1] - z[0]
    N = z.size
    k0 = 2 * np.pi / lambda0
    epsr = (n.astype(complex) ** 2) if np.iscomplexobj(n) else n.astype(float) ** 2
    if np.iscomplexobj(epsr):
        raise NotImplementedError("lossy profiles need the dense solver")
    if pol == "TE":
        di = -2.0 / dz ** 2 + k0 ** 2 * epsr                     # slabModes.m:29-30
        off = np.full(N - 1, 1.0 / dz ** 2)
        w, V = eigh_tridiagonal(di, off, select="i", select_range=(N - nModes, N - 1))
    elif pol == "TM":
        epsH = None if EpsHalf is None else np.asarray(EpsHalf, dtype=float).ravel()
        if epsH is None or epsH.size == 0:
            epsH = 0.5 * (epsr[:-1] + epsr[1:])                # slabModes.m:33-35
        if epsH.size != N - 1:
            raise ValueError("slabModes:epsHalf: EpsHalf needs numel(z)-1 values.")
        up = np.concatenate([1.0 / epsH, [1.0 / epsr[-1]]]) * epsr / dz ** 2   # :38
        lo = np.concatenate([[1.0 / epsr[0]], 1.0 / epsH]) * epsr / dz ** 2    # :39
        di = -(up + lo) + k0 ** 2 * epsr                                          # :40
        # A[k, k+1] = up[k], A[k+1, k] = lo[k+1]; D^-1 A D is symmetric with
        # off-diagonal sqrt(up[k] lo[k+1]) when d[k+1]/d[k] = sqrt(lo[k+1]/up[k]).
        a = up[:-1]
        b = lo[1:]
        off = np.sqrt(a * b)
        w, W = eigh_tridiagonal(di, off, select="i", select_range=(N - nModes, N - 1))
        ratio = np.sqrt(b / a)
        dvec = np.concatenate([[1.0], np.cumprod(ratio)])
        V = W * dvec[:, None]
    else:
        raise ValueError('pol must be "TE" or "TM"')
    order = np.argsort(w)[::-1]
    beta2 = w[order]
    V = V[:, order]
    neff = np.sqrt(beta2.astype(complex)) / k0
    for k in range(nModes):                                      # slabModes.m:49-52
        ip = int(np.argmax(np.abs(V[:, k])))
        V[:, k] = V[:, k] / V[ip, k]
    if np.all(np.abs(neff.imag) == 0):
        neff = neff.real
    return {"neff": neff, "field": V}
