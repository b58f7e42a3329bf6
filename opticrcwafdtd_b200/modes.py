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


# ------------------------------------------------------------ full vector --
def _fwd(n: int, h: float, periodic: bool):
    """Forward difference (f[i+1] - f[i]) / h on n points: zero past the last
    point, or wrapping when periodic."""
    from scipy import sparse
    U = sparse.diags([-np.ones(n), np.ones(n - 1)], [0, 1], shape=(n, n), format="lil")
    if periodic:
        U[n - 1, 0] = 1.0
    return (U.tocsr() / h)


def _wrap_eps(xc, yc, dx, dy, boxes, nBg, hdir, NSub, Lx, x0):
    """epsCellMean with the x samples folded into [x0, x0+Lx): the boxes
    repeat with period Lx along x (geometry.epsCellMean folds its second
    coordinate, so x and y swap roles)."""
    from .geometry import _as_boxes, epsCellMean
    b = _as_boxes(boxes)
    bs = b[:, [2, 3, 0, 1, 4]]
    sdir = {"x": "y", "y": "x"}.get(hdir, hdir)
    return epsCellMean(yc, xc, dy, dx, bs, nBg, sdir, NSub, WrapY=(x0, Lx)).T


def wgModes2D(x, y, nBg: float, boxes, lambda0: float, nModes: int = 1, NGuess=None,
              PeriodicX: bool = False, NSub: int = 4, Eps=None) -> dict:
    """modes = wgModes2D(x, y, nBg, boxes, lambda0, nModes, ...): full-vector
    modes of a waveguide cross-section on the Yee grid, propagating as
    exp(i(beta z - w t)) (the documented method of toolbox/+orf/wgModes2D.m,
    whose implementation is closed).

    x, y: uniform cell centres [um] = the E_z points; E_x, h_y at (i+1/2, j);
    E_y, h_x at (i, j+1/2); h_z at (i+1/2, j+1/2); h = eta0 H.  Eliminating
    E_z and h_z from the curl equations leaves, with U the forward
    differences (zero past the last point; wrapping in x when PeriodicX) and
    V = -U^T,
        beta E_t = P h_t,   beta h_t = Q E_t,   beta^2 E_t = P Q E_t,
        P = (1/k0)[-Ux ez^-1 Vy,  Ux ez^-1 Vx; -Uy ez^-1 Vy,  Uy ez^-1 Vx] + k0[0 I; -I 0]
        Q = (1/k0)[ Vx Uy, -Vx Ux; Vy Uy, -Vy Ux] + k0[0 -ey; ex 0],
    and E_z = i/(k0 ez) (Vx h_y - Vy h_x), h_z = -i/k0 (Ux E_y - Uy E_x).
    eps_x / eps_y are harmonic means along x / y, eps_z the arithmetic mean
    of NSub x NSub samples of the boxes [x1 x2 y1 y2 n] (epsCellMean), unless
    Eps = {"x", "y", "z"} (numel(x) x numel(y) each, e.g. a plane of an FDTD
    grid) gives them.  The nModes eigenvalues of P Q nearest (k0 NGuess)^2
    (default: the largest index present) come from a sparse shift-invert
    solve.

    Returns {"neff" (descending), "Ex", "Ey", "Ez", "Hx", "Hy", "Hz"
    (numel(x) x numel(y) x nModes, complex, scaled so max |E_t| = 1 with that
    entry real and positive), "teFraction" (sum |Ex|^2 / sum |E_t|^2),
    "grid" (coordinates of each component), "eps"}.
    """
    from scipy import sparse
    from scipy.sparse.linalg import eigs

    x = np.asarray(x, dtype=float).ravel()
    y = np.asarray(y, dtype=float).ravel()
    nx, ny = x.size, y.size
    if nx < 2 or ny < 2:
        raise ValueError("wgModes2D:grid: x and y need at least two points.")
    dx, dy = x[1] - x[0], y[1] - y[0]
    k0 = 2 * np.pi / lambda0
    if Eps is not None:
        get = (lambda k: Eps[k]) if isinstance(Eps, dict) else (lambda k: getattr(Eps, k))
        ex, ey, ez = (np.asarray(get(k), dtype=float) for k in ("x", "y", "z"))
        for e in (ex, ey, ez):
            if e.shape != (nx, ny):
                raise ValueError("wgModes2D:eps: Eps.x, .y, .z must be numel(x) x numel(y).")
    elif PeriodicX:
        x0, Lx = x[0] - dx / 2, nx * dx
        ex = _wrap_eps(x + dx / 2, y, dx, dy, boxes, nBg, "x", NSub, Lx, x0)
        ey = _wrap_eps(x, y + dy / 2, dx, dy, boxes, nBg, "y", NSub, Lx, x0)
        ez = _wrap_eps(x, y, dx, dy, boxes, nBg, "none", NSub, Lx, x0)
    else:
        from .geometry import epsCellMean
        ex = epsCellMean(x + dx / 2, y, dx, dy, boxes, nBg, "x", NSub)
        ey = epsCellMean(x, y + dy / 2, dx, dy, boxes, nBg, "y", NSub)
        ez = epsCellMean(x, y, dx, dy, boxes, nBg, "none", NSub)
    N = nx * ny
    nModes = int(nModes)
    if not 1 <= nModes < 2 * N - 1:
        raise ValueError("wgModes2D:nModes: 1 <= nModes < 2 numel(x) numel(y) - 1.")

    # unknowns ordered like a column-major numel(x) x numel(y) array: x fastest
    vec = lambda a: np.asarray(a).ravel(order="F")
    Ix, Iy = sparse.identity(nx, format="csr"), sparse.identity(ny, format="csr")
    Ux = sparse.kron(Iy, _fwd(nx, dx, PeriodicX), format="csr")
    Uy = sparse.kron(_fwd(ny, dy, False), Ix, format="csr")
    Vx, Vy = (-Ux.T).tocsr(), (-Uy.T).tocsr()
    iez = sparse.diags(1.0 / vec(ez))
    I = sparse.identity(N, format="csr")
    P = sparse.bmat([[-Ux @ iez @ Vy, Ux @ iez @ Vx], [-Uy @ iez @ Vy, Uy @ iez @ Vx]]) / k0 \
        + k0 * sparse.bmat([[None, I], [-I, None]])
    Q = sparse.bmat([[Vx @ Uy, -Vx @ Ux], [Vy @ Uy, -Vy @ Ux]]) / k0 \
        + k0 * sparse.bmat([[None, -sparse.diags(vec(ey))], [sparse.diags(vec(ex)), None]])
    P, Q = P.tocsr(), Q.tocsr()
    A = (P @ Q).tocsc()
    ng = float(NGuess) if NGuess is not None else float(np.sqrt(max(ex.max(), ey.max(), ez.max())))
    vals, vecs = eigs(A, k=nModes, sigma=(k0 * ng) ** 2, which="LM")
    beta = np.sqrt(vals.astype(complex))
    neff = beta / k0
    order = np.argsort(-neff.real, kind="stable")
    neff, beta, vecs = neff[order], beta[order], vecs[:, order]

    shp = (nx, ny, nModes)
    F = {k: np.zeros(shp, dtype=complex) for k in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")}
    te = np.zeros(nModes)
    for m in range(nModes):
        Et = vecs[:, m]
        s = Et[int(np.argmax(np.abs(Et)))]
        Et = Et / s
        ht = (Q @ Et) / beta[m]
        Exv, Eyv, hxv, hyv = Et[:N], Et[N:], ht[:N], ht[N:]
        Ezv = 1j / (k0 * vec(ez)) * (Vx @ hyv - Vy @ hxv)
        hzv = -1j / k0 * (Ux @ Eyv - Uy @ Exv)
        for k, v in (("Ex", Exv), ("Ey", Eyv), ("Ez", Ezv), ("Hx", hxv), ("Hy", hyv), ("Hz", hzv)):
            F[k][:, :, m] = v.reshape((nx, ny), order="F")
        px, py = np.sum(np.abs(Exv) ** 2), np.sum(np.abs(Eyv) ** 2)
        te[m] = px / (px + py)
    if np.all(np.abs(neff.imag) <= 1e-12 * np.abs(neff.real)):
        neff = neff.real
    xh, yh = x + dx / 2, y + dy / 2
    grid = {"Ex": (xh, y), "Ey": (x, yh), "Ez": (x, y), "Hx": (x, yh), "Hy": (xh, y), "Hz": (xh, yh)}
    out = {"neff": neff, "teFraction": te, "grid": grid, "eps": {"x": ex, "y": ey, "z": ez}}
    out.update(F)
    return out
