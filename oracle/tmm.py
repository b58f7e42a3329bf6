"""Abeles transfer-matrix method, a numpy restatement of toolbox/+orf/tmm.m:1-72
(open source in the reference) with kzBranch.m:1-9.  TEST COMPARATOR ONLY:
the reference's FDTD tests compare slab R/T against it
(tests/TestFDTD2D.m:34-36, 110; TestFDTD3D.m:224)."""
from __future__ import annotations

import numpy as np


def _kz_branch(kz2):
    # kzBranch.m:6-8: Im(kz) >= 0, and Re(kz) >= 0 when Im(kz) == 0
    kz = np.sqrt(np.asarray(kz2, dtype=complex))
    flip = (kz.imag < 0) | ((kz.imag == 0) & (kz.real < 0))
    return np.where(flip, -kz, kz)


def _admittance(nj, k0, kx, pol):
    kz = _kz_branch(nj ** 2 * k0 ** 2 - kx ** 2)
    q = kz / k0 if pol == "s" else kz / (k0 * nj ** 2)
    return q, kz


def tmm(lambda0, n, d, theta0, pol):
    """out = tmm(lambda0, n, d, theta0, pol) -> dict r, t, R, T, A (Nl x Nt)."""
    lam = np.atleast_1d(np.asarray(lambda0, dtype=float)).reshape(-1, 1)
    n = np.atleast_2d(np.asarray(n, dtype=complex))
    d = np.atleast_1d(np.asarray(d, dtype=float)).ravel()
    th = np.atleast_1d(np.asarray(theta0, dtype=float)).reshape(1, -1)
    M = n.shape[1]
    assert M >= 2 and d.size == M - 2
    if n.shape[0] == 1:
        n = np.repeat(n, lam.shape[0], axis=0)
    k0 = 2 * np.pi / lam
    kx = k0 * n[:, :1].real * np.sin(th)
    q0, _ = _admittance(n[:, :1], k0, kx, pol)
    qs, _ = _admittance(n[:, M - 1:M], k0, kx, pol)
    m11 = np.ones_like(kx, dtype=complex); m12 = np.zeros_like(m11)
    m21 = np.zeros_like(m11); m22 = np.ones_like(m11)
    for j in range(1, M - 1):
        q, kz = _admittance(n[:, j:j + 1], k0, kx, pol)
        delta = kz * d[j - 1]
        c, s = np.cos(delta), np.sin(delta)
        l11, l12, l21, l22 = c, -1j * s / q, -1j * q * s, c
        m11, m12, m21, m22 = (m11 * l11 + m12 * l21, m11 * l12 + m12 * l22,
                              m21 * l11 + m22 * l21, m21 * l12 + m22 * l22)
    Bm = m11 + m12 * qs
    Cm = m21 + m22 * qs
    den = q0 * Bm + Cm
    r = (q0 * Bm - Cm) / den
    t = 2 * q0 / den
    R = np.abs(r) ** 2
    T = qs.real / q0.real * np.abs(t) ** 2
    return {"r": r, "t": t, "R": R, "T": T, "A": 1 - R - T}
