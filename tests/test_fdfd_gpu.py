"""orf.fdfd2D on the device (opticrcwafdtd_b200/fdfd.py, csrc/fdfd.cu) against
the FDFD oracle, on the reference's own physics checks
(tests/TestInverseDesign.m:12-33), and its adjoint gradient."""
import numpy as np
import pytest

import opticrcwafdtd_b200 as orf
from oracle.fdfd import fdfd2D as oracle_fdfd2D
from tests import fdfd_cases

pytestmark = pytest.mark.gpu

# Both sides are direct solves with partial pivoting of the same FP64
# matrix; they differ by rounding amplified by the operator's conditioning.
TOL = 1e-9


def rel(a, b):
    return np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel())


@pytest.mark.parametrize("nx,nz,lossy", [(60, 40, True), (45, 70, False), (300, 150, True), (170, 400, True),
                                         (420, 300, False)])
def test_fdfd_matches_oracle(nx, nz, lossy):
    # blocks of 40 .. 300 points: every cluster shape of the solver, both orientations
    x, z, eps, lam, J, g, npml = fdfd_cases.random_problem(nx, nz, nx + nz, lossy)
    o = orf.fdfd2D(x, z, eps, lam, J, Npml=npml)
    r = oracle_fdfd2D(x, z, eps, lam, J, Npml=npml)
    assert rel(o.E, r.E) <= TOL
    assert rel(o.adjoint(g), r.adjoint(g)) <= TOL
    J2 = np.roll(J, 5, axis=0) * 1j
    assert rel(o.solve(J2), r.solve(J2)) <= TOL
    info = o.info()
    assert info["block"] == min(nx, nz) and info["blocks"] == max(nx, nz)
    o.close()


def test_fdfd_straight_guide_is_exact():
    x, z, epsr, lam, J, m, win = fdfd_cases.straight_guide()
    o = orf.fdfd2D(x, z, epsr, lam, J)
    fdfd_cases.check_straight_guide(o, x, z, m, win)
    r = oracle_fdfd2D(x, z, epsr, lam, J)
    assert rel(o.E, r.E) <= TOL


def test_fdfd_adjoint_gradient_matches_finite_differences():
    x, z, eps, lam, J, g, npml = fdfd_cases.random_problem(50, 36, 8)
    ctx = orf.Context(0)
    o = orf.fdfd2D(x, z, eps, lam, J, Npml=npml, ctx=ctx)
    grad = -o.k0 ** 2 * o.adjoint(g) * o.E
    h = 1e-6
    for (i, k) in ((20, 18), (40, 6), (5, 30)):
        ep, em = eps.copy(), eps.copy()
        ep[i, k] += h
        em[i, k] -= h
        cp = np.sum(g * orf.fdfd2D(x, z, ep, lam, J, Npml=npml, ctx=ctx).E)
        cm = np.sum(g * orf.fdfd2D(x, z, em, lam, J, Npml=npml, ctx=ctx).E)
        assert abs((cp - cm) / (2 * h) - grad[i, k]) <= 1e-6 * max(1.0, abs(grad[i, k]))
    o.close()
    ctx.close()


def test_fdfd_rejects_a_block_above_the_limit():
    x = np.arange(400) * 0.02
    with pytest.raises(orf.OrfError) as ei:
        orf.fdfd2D(x, x, np.ones((400, 400)), 1.55, np.zeros((400, 400)))
    assert ei.value.identifier == "orf:tooLarge"
