"""wgModes2D: the full-vector Yee-grid mode solver (host side).

Pins from the reference's own tests (tests/TestModeSolver2D.m): the slab
limits against slabModes, the degeneracy of a square core and the SOI strip
TE0 index with its grid convergence; plus the discrete Maxwell equations the
returned fields must satisfy."""
import numpy as np
import pytest

from opticrcwafdtd_b200 import slabModes, wgModes2D


def _slab_in_2d():
    """x-invariant Si slab (|y| < 0.11) in SiO2: periodic x, 4 cells
    (TestModeSolver2D.m:11-17)."""
    dy = 0.01
    y = np.arange(-1.5, 1.5 + 1e-9, dy) + dy / 2
    x = (np.arange(4) + 0.5) * 0.05
    m = wgModes2D(x, y, 1.444, [[-np.inf, np.inf, -0.11, 0.11, 3.476]], 1.55, 2, PeriodicX=True)
    return m, y, m["eps"]


def test_slab_limit_te():
    """E_x parallel to the layers = the 1D TE problem on the E_x grid
    (TestModeSolver2D.m:21-27)."""
    m, y, e = _slab_in_2d()
    ref = slabModes(y, np.sqrt(e["x"][0, :]), 1.55, "TE")
    assert abs(m["neff"][0] - ref["neff"][0]) <= 1e-9
    assert m["teFraction"][0] > 0.999


def test_slab_limit_tm():
    """E_y normal to the layers = 1D TM for h_x on the E_y grid, eps_y at the
    points and eps_z between them (TestModeSolver2D.m:29-38)."""
    m, y, e = _slab_in_2d()
    dy = y[1] - y[0]
    ref = slabModes(y + dy / 2, np.sqrt(e["y"][0, :]), 1.55, "TM", EpsHalf=e["z"][0, 1:])
    assert abs(m["neff"][1] - ref["neff"][0]) <= 2e-7     # the wall treatment differs at the edge
    assert m["teFraction"][1] < 1e-3


def test_square_core_is_degenerate():
    """90-degree symmetry: the two fundamental modes share neff, and the pair
    spans both polarisations (TestModeSolver2D.m:40-47)."""
    d = 0.01
    c = (np.arange(-100, 100) + 0.5) * d
    m = wgModes2D(c, c, 1.444, [[-0.2, 0.2, -0.2, 0.2, 3.476]], 1.55, 2)
    assert abs(m["neff"][0] - m["neff"][1]) <= 1e-6
    assert abs(np.sum(m["teFraction"]) - 1.0) <= 1e-3


def test_soi_strip_te0():
    """500 x 220 nm Si strip in SiO2 at 1550 nm: TE0 near 2.44, refining the
    grid changes neff by < 3e-3 (TestModeSolver2D.m:49-64)."""
    n = []
    for k in (1, 2):
        d = 0.02 / k
        x = (np.arange(-round(1.5 / d), round(1.5 / d)) + 0.5) * d
        y = (np.arange(-round(1.2 / d), round(1.2 / d)) + 0.5) * d
        m = wgModes2D(x, y, 1.444, [[-0.25, 0.25, -0.11, 0.11, 3.476]], 1.55, 2)
        n.append(m["neff"][int(np.argmax(m["teFraction"]))])
    assert 2.40 < n[1] < 2.48
    assert abs(n[1] - n[0]) < 3e-3


def _ops(nx, ny, dx, dy, periodic_x=False):
    """The difference operators on the column-major numel(x) x numel(y) layout."""
    from scipy import sparse
    def fwd(n, h, per):
        U = sparse.diags([-np.ones(n), np.ones(n - 1)], [0, 1], shape=(n, n), format="lil")
        if per:
            U[n - 1, 0] = 1.0
        return U.tocsr() / h
    Ux = sparse.kron(sparse.identity(ny), fwd(nx, dx, periodic_x), format="csr")
    Uy = sparse.kron(fwd(ny, dy, False), sparse.identity(nx), format="csr")
    return Ux, Uy, -Ux.T, -Uy.T


def test_modes_satisfy_the_discrete_maxwell_equations():
    """Every returned mode solves the six Yee-grid curl equations with
    d/dz = i beta (h = eta0 H):
        Uy Ez - i b Ey = i k0 hx,   i b Ex - Ux Ez = i k0 hy,   Ux Ey - Uy Ex = i k0 hz,
        Vy hz - i b hy = -i k0 ex Ex,   i b hx - Vx hz = -i k0 ey Ey,   Vx hy - Vy hx = -i k0 ez Ez."""
    d = 0.02
    x = (np.arange(-40, 40) + 0.5) * d
    y = (np.arange(-30, 30) + 0.5) * d
    lam = 1.55
    m = wgModes2D(x, y, 1.444, [[-0.25, 0.25, -0.11, 0.11, 3.476], [-0.6, 0.6, -0.6, -0.11, 2.0]], lam, 3)
    k0 = 2 * np.pi / lam
    Ux, Uy, Vx, Vy = _ops(x.size, y.size, d, d)
    v = lambda a: a.ravel(order="F")
    ex, ey, ez = (v(m["eps"][k]) for k in "xyz")
    for q in range(3):
        b = k0 * m["neff"][q]
        Ex, Ey, Ez, Hx, Hy, Hz = (v(m[k][:, :, q]) for k in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"))
        scale = k0 * max(np.abs(Ex).max(), np.abs(Ey).max())
        res = [Uy @ Ez - 1j * b * Ey - 1j * k0 * Hx,
               1j * b * Ex - Ux @ Ez - 1j * k0 * Hy,
               Ux @ Ey - Uy @ Ex - 1j * k0 * Hz,
               Vy @ Hz - 1j * b * Hy + 1j * k0 * ex * Ex,
               1j * b * Hx - Vx @ Hz + 1j * k0 * ey * Ey,
               Vx @ Hy - Vy @ Hx + 1j * k0 * ez * Ez]
        for r in res:
            assert np.max(np.abs(r)) <= 1e-10 * scale


def test_normalisation_and_eps_option():
    """max |E_t| = 1 on a real positive entry; handing the solver its own eps
    (the Eps option, e.g. a plane of an FDTD grid) reproduces the modes."""
    d = 0.02
    x = (np.arange(-40, 40) + 0.5) * d
    y = (np.arange(-30, 30) + 0.5) * d
    boxes = [[-0.25, 0.25, -0.11, 0.11, 3.476]]
    m = wgModes2D(x, y, 1.444, boxes, 1.55, 2)
    for q in range(2):
        Et = np.concatenate([m["Ex"][:, :, q].ravel(), m["Ey"][:, :, q].ravel()])
        k = int(np.argmax(np.abs(Et)))
        assert abs(Et[k] - 1.0) < 1e-12
    m2 = wgModes2D(x, y, 9.9, np.zeros((0, 5)), 1.55, 2, Eps=m["eps"])
    assert np.allclose(m2["neff"], m["neff"], rtol=0, atol=1e-11)
    assert m["grid"]["Hz"][0][0] == pytest.approx(x[0] + d / 2)


def test_periodic_x_folds_boxes_across_the_edge():
    """With PeriodicX a box that leaves the domain re-enters on the other
    side: shifting it by the period changes nothing."""
    d = 0.02
    x = (np.arange(40) + 0.5) * d          # period 0.8
    y = (np.arange(-30, 30) + 0.5) * d
    a = wgModes2D(x, y, 1.444, [[-0.1, 0.2, -0.11, 0.11, 3.476]], 1.55, 1, PeriodicX=True)
    b = wgModes2D(x, y, 1.444, [[0.7, 1.0, -0.11, 0.11, 3.476]], 1.55, 1, PeriodicX=True)
    for k in "xyz":
        assert np.allclose(a["eps"][k], b["eps"][k], rtol=0, atol=1e-12)
    assert abs(a["neff"][0] - b["neff"][0]) < 1e-10
