"""Pins of the FP64 CPU oracle (CPU only).

The reference's hot path lives in MRCPP, which is not vendored; the oracle restates the published
method and is pinned here by (1) exact analytic results (Poisson and Helmholtz potentials of a
Gaussian charge, exact hydrogenic Coulomb integrals) and (2) the reference's own known-answer
tests, tests/qmoperators/coulomb_operator.cpp:76-82 and tests/qmfunctions/orbital*.cpp.
"""
import json
import os

import numpy as np
import pytest
from scipy import integrate
from scipy.special import erf, erfcx

HERE = os.path.dirname(os.path.abspath(__file__))
WORLD = (-2, (-5, -5, -5), (10, 10, 10))


def helmholtz_gaussian(r, alpha, mu):
    """int exp(-mu|r-r'|)/|r-r'| (alpha/pi)^{3/2} exp(-alpha r'^2) dr' (closed form, stable)."""
    sa = np.sqrt(alpha)
    x1 = mu / (2 * sa) - sa * r
    x2 = mu / (2 * sa) + sa * r
    g = np.exp(-alpha * r * r)
    t2 = erfcx(x2) * g
    if x1 > 0:
        t1 = erfcx(x1) * g
    else:
        from scipy.special import erfc

        t1 = np.exp(mu * mu / (4 * alpha) - mu * r) * erfc(x1)
    return (t1 - t2) / (2 * r)


@pytest.mark.parametrize("basis", [0, 1])
@pytest.mark.parametrize("order", [3, 5, 7, 9, 11])
def test_filters_orthogonal(oracle_mod, basis, order):
    m = oracle_mod.MultiResolutionAnalysis(*WORLD, order, 10, basis=basis)
    F = m.filter()
    assert np.abs(F @ F.T - np.eye(2 * (order + 1))).max() < 1e-12


def _phi_interp(j, x, k):
    xg, wg = np.polynomial.legendre.leggauss(k)
    xg, wg = 0.5 * (xg + 1), 0.5 * wg
    v = 0.0
    for i in range(k):
        c = np.zeros(i + 1)
        c[i] = 1
        v = v + (2 * i + 1) * np.polynomial.legendre.legval(2 * xg[j] - 1, c) * np.polynomial.legendre.legval(2 * x - 1, c)
    return v * np.sqrt(wg[j])


@pytest.mark.parametrize("alpha,n,l", [(3.0, 0, 0), (3.0, 0, 1), (50.0, 1, 0), (0.01, -2, 2)])
def test_operator_scaling_matrix_quadrature(oracle_mod, alpha, n, l):
    m = oracle_mod.MultiResolutionAnalysis(*WORLD, 5, 10)
    op = oracle_mod.PoissonOperator(m, 1e-3)
    T = op.scaling_matrix(alpha, n, l)
    i, j = 2, 4
    f = lambda v, u: _phi_interp(i, u, 6) * _phi_interp(j, v, 6) * np.exp(-alpha * 4.0 ** (-n) * (u - v + l) ** 2)
    ref = 2.0 ** (-n) * integrate.dblquad(f, 0, 1, 0, 1, epsabs=1e-13, epsrel=1e-12)[0]
    assert abs(T[i, j] - ref) < 1e-13


def test_kernel_expansion_accuracy(oracle_mod):
    m = oracle_mod.MultiResolutionAnalysis(*WORLD, 5, 12)
    for mu, prec in [(0.0, 1e-5), (1.5, 1e-5)]:
        op = oracle_mod.ConvolutionOperator(m, mu, prec)
        a, b = op.terms()
        eps = 0.1 * prec  # expansion accuracy the operators are built with
        r = np.geomspace(1e-4, 60.0, 300)
        approx = np.array([(b * np.exp(-a * x * x)).sum() for x in r])
        exact = np.exp(-mu * r) / r
        # |error| <= a few eps times the Poisson kernel (capped at r = 1); for mu = 0 this is a
        # relative error bound on the whole range
        assert np.all(np.abs(approx - exact) <= 2 * eps * np.maximum(1.0 / r, 1.0))
        if mu == 0.0:
            assert np.max(np.abs(approx - exact) / exact) < 1.2 * eps


@pytest.mark.parametrize("order,prec,tol", [(5, 1e-3, 2e-3), (7, 1e-5, 2e-5)])
def test_poisson_of_gaussian_matches_erf(oracle_mod, order, prec, tol):
    O = oracle_mod
    m = O.MultiResolutionAnalysis(*WORLD, order, 14)
    alpha, c = 10.0, np.array([0.1, -0.2, 0.3])
    inp = O.FunctionTree(m)
    O.project(prec, inp, O.gauss_params([(alpha / np.pi) ** 1.5], [alpha], [c]))
    assert abs(inp.square_norm() - (alpha / (2 * np.pi)) ** 1.5) < 10 * prec
    out = O.FunctionTree(m)
    O.apply(prec, out, O.PoissonOperator(m, prec), inp)
    rng = np.random.default_rng(0)
    err = 0.0
    for _ in range(200):
        r = rng.uniform(-4, 4, 3) + c
        d = np.linalg.norm(r - c)
        err = max(err, abs(out.evalf(r) - erf(np.sqrt(alpha) * d) / d))
    vmax = 2 * np.sqrt(alpha / np.pi)
    assert err < tol * vmax


@pytest.mark.parametrize("mu", [0.7, 2.5])
def test_helmholtz_of_gaussian_matches_closed_form(oracle_mod, mu):
    O = oracle_mod
    prec = 1e-5
    m = O.MultiResolutionAnalysis(*WORLD, 7, 14)
    alpha, c = 8.0, np.array([-0.3, 0.2, 0.1])
    inp = O.FunctionTree(m)
    O.project(prec, inp, O.gauss_params([(alpha / np.pi) ** 1.5], [alpha], [c]))
    out = O.FunctionTree(m)
    O.apply(prec, out, O.HelmholtzOperator(m, mu, prec), inp)
    rng = np.random.default_rng(1)
    err = 0.0
    vmax = helmholtz_gaussian(1e-6, alpha, mu)
    for _ in range(200):
        r = rng.uniform(-3, 3, 3) + c
        d = np.linalg.norm(r - c)
        err = max(err, abs(out.evalf(r) - helmholtz_gaussian(d, alpha, mu)))
    assert err < 3e-5 * vmax


def _kat_setup(O, prec, order):
    kat = json.load(open(os.path.join(HERE, "golden", "reference_kats.json")))
    w = kat["world"]
    m = O.MultiResolutionAnalysis(w["min_scale"], w["corner"], w["boxes"], order, w["max_depth"])
    orbs = [tuple(o) for o in kat["orbitals"]]
    rho = O.FunctionTree(m)
    O.project(prec, rho, O.hydrogen_params([(2.0, o, o) for o in orbs]))
    V = O.FunctionTree(m)
    O.apply(prec / np.sqrt(rho.square_norm()), V, O.PoissonOperator(m, prec), rho)  # CoulombPotential.cpp:80-85
    return kat, m, orbs, V


def _expect(O, m, V, a, b):
    d = O.FunctionTree(m)
    O.project(1e-7, d, O.hydrogen_params([(1.0, a, b)]))
    return O.dot(d, V)


def test_coulomb_kat_converges_to_analytic(oracle_mod):
    """The reference's E_P quantities converge to the exact hydrogenic Coulomb integrals."""
    O = oracle_mod
    kat, m, orbs, V = _kat_setup(O, 1e-5, 7)
    for key, expr in kat["analytic_E_P"].items():
        i, j = map(int, key.split(","))
        exact = eval(expr)  # rational constants from the fixture
        val = _expect(O, m, V, orbs[i], orbs[j])
        assert abs(val - exact) / exact < 1e-4, (key, val, exact)


def test_coulomb_kat_reference_values_at_prec_1e3(oracle_mod):
    """At the reference's own setting (prec 1e-3, order 5) the oracle agrees with the KAT values of
    tests/qmoperators/coulomb_operator.cpp:76-82 to precision level.  Those values are MRCPP's
    output at that precision and differ from the exact integrals by up to 1.3% (0,0) and 6% (0,1)
    themselves, so they pin the apply only to a few percent; the analytic pin above is the tight one."""
    O = oracle_mod
    kat, m, orbs, V = _kat_setup(O, 1e-3, 5)
    for key, ref in kat["coulomb_operator_E_P"].items():
        i, j = map(int, key.split(","))
        val = _expect(O, m, V, orbs[i], orbs[j])
        tol = 0.12 if i != j else 0.03
        assert abs(val - ref) / ref < tol, (key, val, ref)


def _hessian_setup(O, prec, order):
    """Response Coulomb potential of tests/qmoperators/coulomb_hessian.cpp: V = P[rho_1] with
    rho_1 = 4 (1s 2s + 2s 2p1) (density_utils.cpp:226-260, paired occupation 2, X = Y)."""
    kat = json.load(open(os.path.join(HERE, "golden", "reference_kats.json")))
    w = kat["world"]
    m = O.MultiResolutionAnalysis(w["min_scale"], w["corner"], w["boxes"], order, w["max_depth"])
    phi = [tuple(o) for o in kat["hessian"]["phi"]]
    x = [tuple(o) for o in kat["hessian"]["x"]]
    rho = O.FunctionTree(m)
    O.project(prec, rho, O.hydrogen_params([(4.0, p, q) for p, q in zip(phi, x)]))
    V = O.FunctionTree(m)
    O.apply(prec / np.sqrt(rho.square_norm()), V, O.PoissonOperator(m, prec), rho)  # CoulombPotential.cpp:80-85
    return kat, m, phi, V


def test_coulomb_hessian_kat_converges_to_analytic(oracle_mod):
    """tests/qmoperators/coulomb_hessian.cpp:95-98: the E_P quantities converge to the exact hydrogenic
    integrals 4[1s1s|1s2s], 4[1s2s|1s2s], 4[2s2s|1s2s] (to 1e-4 at order 9, prec 1e-6)."""
    O = oracle_mod
    kat, m, phi, V = _hessian_setup(O, 1e-6, 9)
    for key, expr in kat["analytic_hessian_E_P"].items():
        i, j = map(int, key.split(","))
        exact = eval(expr)  # closed forms from the fixture
        val = _expect(O, m, V, phi[i], phi[j])
        assert abs(val - exact) / exact < 1e-4, (key, val, exact)


def test_coulomb_hessian_kat_reference_values(oracle_mod):
    """The reference's E_P values (MRCPP at prec 1e-3) lie within 0.5 % of the converged oracle values
    (they are that precision's approximation of the exact integrals: 0.28 % / 0.46 % / 0.47 % away);
    at the reference's own setting (order 5, prec 1e-3) the oracle agrees with them to 8 %."""
    O = oracle_mod
    kat, m, phi, V = _hessian_setup(O, 1e-5, 7)
    for key, ref in kat["coulomb_hessian_E_P"].items():
        i, j = map(int, key.split(","))
        val = _expect(O, m, V, phi[i], phi[j])
        assert abs(val - ref) / ref < 5e-3, (key, val, ref)
    kat, m, phi, V = _hessian_setup(O, 1e-3, 5)
    for key, ref in kat["coulomb_hessian_E_P"].items():
        i, j = map(int, key.split(","))
        val = _expect(O, m, V, phi[i], phi[j])
        assert abs(val - ref) / ref < 0.08, (key, val, ref)


def test_projected_hydrogen_orbitals_are_normalised(oracle_mod):
    """tests/qmfunctions/orbital_vector.cpp:145: projected hydrogen orbitals have norm 1 (Approx)."""
    O = oracle_mod
    kat = json.load(open(os.path.join(HERE, "golden", "reference_kats.json")))
    w = kat["world"]
    m = O.MultiResolutionAnalysis(w["min_scale"], w["corner"], w["boxes"], w["order"], w["max_depth"])
    for o in kat["orbitals"]:
        t = O.FunctionTree(m)
        O.project(w["prec"], t, O.hydrogen_params([(1.0, tuple(o), None)]))
        assert abs(np.sqrt(t.square_norm()) - 1.0) < 1.2e-5


def test_density_integrates_to_electron_count(oracle_mod):
    """tests/qmfunctions/density.cpp:71: the total density integrates to the electron count."""
    O = oracle_mod
    kat = json.load(open(os.path.join(HERE, "golden", "reference_kats.json")))
    w = kat["world"]
    m = O.MultiResolutionAnalysis(w["min_scale"], w["corner"], w["boxes"], w["order"], w["max_depth"])
    occ = [(1, (1, 0, 0)), (1, (2, 0, 0)), (1, (2, 1, 0)), (1, (2, 1, 1)), (1, (2, 1, 2)), (2, (1, 0, 0))]
    rho = O.FunctionTree(m)
    O.project(w["prec"], rho, O.hydrogen_params([(float(c), o, o) for c, o in occ]))
    one = O.FunctionTree(m)
    O.project(w["prec"], one, O.gauss_params([1.0], [1e-12], [(0.0, 0.0, 0.0)]))
    assert abs(O.dot(rho, one) - 7.0) < 7.0 * 1.2e-5


def test_oracle_golden_regression(oracle_mod):
    """Small fixed case against the committed fixture (tests/golden/make_golden.py)."""
    O = oracle_mod
    g = np.load(os.path.join(HERE, "golden", "oracle_small.npz"))
    m = O.MultiResolutionAnalysis(*WORLD, 5, 10)
    inp = O.FunctionTree(m)
    O.project(1e-3, inp, (int(g["ftype"]), g["params"]))
    out = O.FunctionTree(m)
    O.apply(1e-3, out, O.PoissonOperator(m, 1e-3), inp)
    ex = out.export()
    keys = sorted((int(d), *map(int, t)) for d, t in zip(ex["depth"], ex["trans"]))
    assert np.array_equal(np.array(keys), g["out_keys"])
    assert abs(out.square_norm() - float(g["out_norm2"])) < 1e-10 * float(g["out_norm2"])


def test_oracle_multiply_gaussian_product(oracle_mod):
    """The MW product of two Gaussians against the closed form: the norm of
    exp(-a1|r-c1|^2) exp(-a2|r-c2|^2), point values, and the union-grid form (maxIter 0)."""
    O = oracle_mod
    m = O.MultiResolutionAnalysis(*WORLD, 5, 12)
    a1, c1, a2, c2 = 2.0, np.array([0.1, -0.2, 0.3]), 3.0, np.array([-0.3, 0.2, 0.1])
    A, B = O.FunctionTree(m), O.FunctionTree(m)
    O.project(1e-4, A, O.gauss_params([1.0], [a1], [c1]))
    O.project(1e-4, B, O.gauss_params([1.0], [a2], [c2]))
    exact2 = (np.pi / (2 * a1 + 2 * a2)) ** 1.5 * np.exp(-2 * a1 * a2 / (a1 + a2) * np.sum((c1 - c2) ** 2))
    P = O.FunctionTree(m)
    O.multiply(1e-4, P, 1.0, A, B)
    assert abs(P.square_norm() - exact2) < 1e-8 * exact2
    rng = np.random.default_rng(0)
    for _ in range(50):
        r = rng.uniform(-1.0, 1.0, 3)
        ex = np.exp(-a1 * np.sum((r - c1) ** 2) - a2 * np.sum((r - c2) ** 2))
        assert abs(P.evalf(r) - ex) < 1e-5
    U = O.FunctionTree(m)
    O.build_grid(U, A)
    O.build_grid(U, B)
    ka = {(int(d), *map(int, t)) for e in (A.export(False), B.export(False)) for d, t in zip(e["depth"], e["trans"])}
    eu = U.export(False)
    assert {(int(d), *map(int, t)) for d, t in zip(eu["depth"], eu["trans"])} == ka
    O.multiply(-1.0, U, 2.0, A, B, 0)
    assert U.nnodes() == len(ka)
    assert abs(U.square_norm() - 4.0 * exact2) < 1e-8 * exact2
