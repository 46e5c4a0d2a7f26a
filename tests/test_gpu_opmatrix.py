"""The library's own operator matrices against quadrature that shares no code with it or with the
oracle: T^n(l) entries of exp(-alpha x^2) between interpolating scaling functions by scipy double
quadrature, and NS matrices by the two-scale composition of such T's in numpy.  The oracle restates the
same construction, so parity between the GPU path and the oracle alone could not catch a defect
common to both; these checks can.  (Needs the library, which needs a CUDA device to create a world.)
"""
import numpy as np
import pytest
from scipy import integrate

pytestmark = pytest.mark.gpu

WORLD = (-2, (-5, -5, -5), (10, 10, 10))


def phi_interp(j, x, k):
    """interpolating scaling function j of order k - 1 on [0, 1] (Legendre-Gauss nodes), numpy"""
    xg, wg = np.polynomial.legendre.leggauss(k)
    xg, wg = 0.5 * (xg + 1), 0.5 * wg
    v = 0.0
    for i in range(k):
        c = np.zeros(i + 1)
        c[i] = 1
        v = v + (2 * i + 1) * np.polynomial.legendre.legval(2 * xg[j] - 1, c) * np.polynomial.legendre.legval(2 * x - 1, c)
    return v * np.sqrt(wg[j])


def t_quad(alpha, n, l, i, j, k):
    f = lambda v, u: phi_interp(i, u, k) * phi_interp(j, v, k) * np.exp(-alpha * 4.0 ** (-n) * (u - v + l) ** 2)
    return 2.0 ** (-n) * integrate.dblquad(f, 0, 1, 0, 1, epsabs=1e-13, epsrel=1e-12)[0]


@pytest.mark.parametrize("alpha,n,l,i,j", [(3.0, 0, 0, 2, 4), (3.0, 0, 1, 0, 5), (50.0, 1, 0, 5, 1), (0.01, -2, 2, 3, 3),
                                           (700.0, 2, -1, 1, 4)])
def test_scaling_matrix_against_dblquad(gpu_mod, alpha, n, l, i, j):
    G = gpu_mod
    m = G.MultiResolutionAnalysis(*WORLD, 5, 10)
    op = G.PoissonOperator(m, 1e-3)
    T = op.scaling_matrix(alpha, n, l)
    assert abs(T[i, j] - t_quad(alpha, n, l, i, j, 6)) < 1e-13


def test_ns_matrix_against_two_scale_composition(gpu_mod):
    """NS(n, l) = F [[T(2l) T(2l-1)]; [T(2l+1) T(2l)]]_{n+1} F^T from quadrature T's; F is checked
    orthogonal and to reproduce the scaling functions' two-scale relation independently."""
    G = gpu_mod
    order, k = 3, 4
    m = G.MultiResolutionAnalysis(*WORLD, order, 10)
    op = G.PoissonOperator(m, 1e-3)
    F = m.filter()
    assert np.abs(F @ F.T - np.eye(2 * k)).max() < 1e-12
    # the scaling rows of F carry phi_j(x) on the two children: phi_j(x) = sqrt(2) sum_c H_c phi(2x - c)
    xs = np.linspace(0.01, 0.99, 7)
    for j in range(k):
        for x in xs:
            c = 0 if x < 0.5 else 1
            lhs = phi_interp(j, x, k)
            rhs = np.sqrt(2.0) * sum(F[j, c * k + q] * phi_interp(q, 2 * x - c, k) for q in range(k))
            assert abs(lhs - rhs) < 1e-12
    alpha, beta = op.terms()
    mi = len(alpha) // 2
    for n, l in [(0, 0), (1, 1), (2, -1)]:
        NS = op.ns_matrix(mi, n, l)
        T = {d: np.array([[t_quad(alpha[mi], n + 1, d, i, j, k) for j in range(k)] for i in range(k)])
             for d in (2 * l - 1, 2 * l, 2 * l + 1)}
        mid = np.block([[T[2 * l], T[2 * l - 1]], [T[2 * l + 1], T[2 * l]]])
        ref = F @ mid @ F.T
        assert np.abs(NS - ref).max() < 1e-12 * max(1.0, np.abs(ref).max())
