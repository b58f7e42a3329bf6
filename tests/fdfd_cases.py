"""FDFD problems shared by the oracle and GPU tests."""
import numpy as np


def straight_guide():
    """tests/TestInverseDesign.m:12-24 (straightWaveguideIsExact); see
    workloads.fdfd_straight_guide.  Returns (x, z, epsr, lam, J, m, win)."""
    from opticrcwafdtd_b200 import workloads
    return workloads.fdfd_straight_guide()


def check_straight_guide(o, x, z, m, win):
    """The reference's checks (tests/TestInverseDesign.m:25-32): lossless
    guide (1e-5), even split both ways (1e-4), phase velocity of the Yee
    dispersion of the slab mode (1e-5)."""
    d = x[1] - x[0]
    iz = np.arange(1, z.size + 1)
    P4 = o.fluxX(round(4 / d) + 1, iz)
    P8 = o.fluxX(round(8 / d) + 1, iz)
    assert abs(P8 / P4 - 1) <= 1e-5
    assert abs(o.fluxX(round(1 / d) + 1, iz) / P4 + 1) <= 1e-4
    k = int(np.argmax(np.abs(m["field"][:, 0]))) + int(np.nonzero(win)[0][0])
    xr = np.arange(round(4 / d), round(8 / d) + 1)
    ph = np.polyfit(x[xr], np.unwrap(np.angle(o.E[xr, k])), 1)
    neff = float(np.atleast_1d(m["neff"])[0])
    nYee = (2 / d) * np.arcsin(neff * o.k0 * d / 2) / o.k0
    assert abs(ph[0] / o.k0 - nYee) <= 1e-5


def random_problem(nx, nz, seed, lossy=True, npml=(8, 6)):
    """Random two-material grid (optionally lossy), a line current, a random
    adjoint source.  Returns (x, z, eps, lam, J, g, npml)."""
    rng = np.random.default_rng(seed)
    d = 0.03
    x = np.arange(nx) * d
    z = np.arange(nz) * d
    eps = 1.0 + 10.0 * (rng.random((nx, nz)) < 0.3)
    if lossy:
        eps = eps + 0.05j * rng.random((nx, nz))
    J = np.zeros((nx, nz), dtype=np.complex128)
    J[nx // 3, nz // 4: 3 * nz // 4] = 1.0 + 0.3j
    g = rng.standard_normal((nx, nz)) + 1j * rng.standard_normal((nx, nz))
    return x, z, eps, 1.3, J, g, npml
