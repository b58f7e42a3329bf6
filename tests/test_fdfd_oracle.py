"""The FDFD oracle (oracle/fdfd.py) pinned on the reference's own checks of
orf.fdfd2D (tests/TestInverseDesign.m:12-33) and on the adjoint identity."""
import numpy as np

from oracle.fdfd import fdfd2D, operator
from tests import fdfd_cases


def test_oracle_straight_guide_is_exact():
    x, z, epsr, lam, J, m, win = fdfd_cases.straight_guide()
    o = fdfd2D(x, z, epsr, lam, J)
    fdfd_cases.check_straight_guide(o, x, z, m, win)


def test_oracle_adjoint_gradient_matches_finite_differences():
    # c = sum(g .* E):  dc/deps = -k0^2 lam .* E with A.' lam = g (fdfd2D.m:13-15)
    x, z, eps, lam, J, g, npml = fdfd_cases.random_problem(30, 24, 3)
    o = fdfd2D(x, z, eps, lam, J, Npml=npml)
    grad = -o.k0 ** 2 * o.adjoint(g) * o.E
    h = 1e-6
    for (i, k) in ((10, 12), (20, 5), (3, 20)):
        ep, em = eps.copy(), eps.copy()
        ep[i, k] += h
        em[i, k] -= h
        cp = np.sum(g * fdfd2D(x, z, ep, lam, J, Npml=npml).E)
        cm = np.sum(g * fdfd2D(x, z, em, lam, J, Npml=npml).E)
        fd = (cp - cm) / (2 * h)
        assert abs(fd - grad[i, k]) <= 1e-6 * max(1.0, abs(grad[i, k]))


def test_oracle_operator_is_the_documented_stencil():
    # a row away from the PML: the plain 5-point Laplacian plus k0^2 eps
    x, z, eps, lam, J, g, npml = fdfd_cases.random_problem(30, 24, 4)
    d, k0 = x[1] - x[0], 2 * np.pi / lam
    A = operator(30, 24, d, eps, k0, npml).tocsr()
    i, k = 15, 12
    r = i + 30 * k
    row = A.getrow(r).toarray().ravel()
    assert np.isclose(row[r], -4 / d ** 2 + k0 ** 2 * eps[i, k])
    for q in (r - 1, r + 1, r - 30, r + 30):
        assert np.isclose(row[q], 1 / d ** 2)
    assert np.count_nonzero(row) == 5
