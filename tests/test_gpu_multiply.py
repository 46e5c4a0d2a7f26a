"""GPU parity of the pointwise product (mrcpp::multiply / square / build_grid contract) against the
FP64 CPU oracle, an analytic check, and the exchange pair pipeline (pair product on the union grid,
then a Poisson apply) of reference src/qmoperators/two_electron/ExchangePotential.cpp:131-137.

Bar: integer tree structure identical; FP64 coefficients within 1e-10 of the largest coefficient.
Factors are projected on the GPU and loaded unchanged into the oracle.
"""
import numpy as np
import pytest

from test_gpu_parity import WORLD, assert_same_tree, pair, to_oracle

pytestmark = pytest.mark.gpu


def gauss(G, a, c, coef=1.0):
    return G.gauss_params([coef], [a], [c])


A1, C1 = 2.0, np.array([0.1, -0.2, 0.3])
A2, C2 = 3.0, np.array([-0.3, 0.2, 0.1])


def product_norm2(a1, c1, a2, c2):
    """|| exp(-a1|r-c1|^2) exp(-a2|r-c2|^2) ||^2"""
    return (np.pi / (2 * a1 + 2 * a2)) ** 1.5 * np.exp(-2 * a1 * a2 / (a1 + a2) * np.sum((c1 - c2) ** 2))


def factors(G, O, mg, mo, prec):
    ag, bg = G.FunctionTree(mg), G.FunctionTree(mg)
    G.project(prec, ag, gauss(G, A1, C1))
    G.project(prec, bg, gauss(G, A2, C2))
    return ag, bg, to_oracle(O, mo, ag), to_oracle(O, mo, bg)


@pytest.mark.parametrize("order,prec", [(5, 1e-4), (7, 1e-5), (9, 1e-6)])
def test_multiply_adaptive_parity(gpu_mod, oracle_mod, order, prec):
    G, O = gpu_mod, oracle_mod
    mg, mo = pair(G, O, order)
    ag, bg, ao, bo = factors(G, O, mg, mo, prec)
    pg, po = G.FunctionTree(mg), O.FunctionTree(mo)
    G.multiply(prec, pg, 0.7, ag, bg)
    O.multiply(prec, po, 0.7, ao, bo)
    assert_same_tree(pg.export(), po.export())
    assert abs(pg.square_norm() - po.square_norm()) < 1e-12 * po.square_norm()
    exact = 0.49 * product_norm2(A1, C1, A2, C2)
    assert abs(pg.square_norm() - exact) < 1e3 * prec * exact


def test_multiply_union_grid_parity(gpu_mod, oracle_mod):
    """prec < 0 form of qmfunction::multiply_real: union grid, no refinement (maxIter 0)"""
    G, O = gpu_mod, oracle_mod
    mg, mo = pair(G, O, 7)
    ag, bg, ao, bo = factors(G, O, mg, mo, 1e-5)
    pg, po = G.FunctionTree(mg), O.FunctionTree(mo)
    G.build_grid(pg, ag)
    G.build_grid(pg, bg)
    O.build_grid(po, ao)
    O.build_grid(po, bo)
    assert pg.nnodes() == po.nnodes()
    G.multiply(-1.0, pg, 1.0, ag, bg, 0)
    O.multiply(-1.0, po, 1.0, ao, bo, 0)
    assert_same_tree(pg.export(), po.export())
    union = {(int(d), *map(int, t)) for e in (ag.export(False), bg.export(False)) for d, t in zip(e["depth"], e["trans"])}
    got = {(int(d), *map(int, t)) for d, t in zip(pg.export(False)["depth"], pg.export(False)["trans"])}
    assert got == union


def test_multiply_against_projected_product(gpu_mod):
    """||a b - P[exact product]|| small, with the exact product projected at the same precision"""
    G = gpu_mod
    mg = G.MultiResolutionAnalysis(*WORLD, 7, 14)
    prec = 1e-6
    ag, bg = G.FunctionTree(mg), G.FunctionTree(mg)
    G.project(prec, ag, gauss(G, A1, C1))
    G.project(prec, bg, gauss(G, A2, C2))
    pg = G.FunctionTree(mg)
    G.multiply(prec, pg, 1.0, ag, bg)
    # exp(-a1|r-c1|^2 - a2|r-c2|^2) = K exp(-(a1+a2)|r-R|^2)
    a = A1 + A2
    R = (A1 * C1 + A2 * C2) / a
    K = np.exp(-A1 * A2 / a * np.sum((C1 - C2) ** 2))
    eg = G.FunctionTree(mg)
    G.project(prec, eg, G.gauss_params([K], [a], [tuple(R)]))
    n_p, n_e, x = pg.square_norm(), eg.square_norm(), G.dot(pg, eg)
    err = np.sqrt(max(n_p + n_e - 2 * x, 0.0) / n_e)
    assert err < 20 * prec, err


def test_square_and_batched_equal_single(gpu_mod):
    G = gpu_mod
    mg = G.MultiResolutionAnalysis(*WORLD, 5, 14)
    prec = 1e-4
    ts = []
    for a, c in ((A1, C1), (A2, C2), (1.5, np.array([0.4, 0.0, -0.2]))):
        t = G.FunctionTree(mg)
        G.project(prec, t, gauss(G, a, c))
        ts.append(t)
    sq, mu = G.FunctionTree(mg), G.FunctionTree(mg)
    G.square(prec, sq, ts[0])
    G.multiply(prec, mu, 1.0, ts[0], ts[0])
    assert_same_tree(sq.export(), mu.export(), tol=0.0)
    pairs = [(0, 1), (1, 2), (0, 2)]
    coefs = [1.0, -2.0, 0.5]
    single = []
    for (i, j), c in zip(pairs, coefs):
        t = G.FunctionTree(mg)
        G.multiply(prec, t, c, ts[i], ts[j])
        single.append(t)
    outs = [G.FunctionTree(mg) for _ in pairs]
    G.multiply_batched(prec, outs, coefs, [ts[i] for i, _ in pairs], [ts[j] for _, j in pairs])
    for a, b in zip(outs, single):
        assert_same_tree(a.export(), b.export(), tol=0.0)


def test_exchange_pair_then_poisson(gpu_mod, oracle_mod):
    """phi_i phi_j on the union grid, then P[phi_i phi_j]: both steps against the oracle"""
    G, O = gpu_mod, oracle_mod
    from mrchem_b200 import workloads as W

    order, prec = 7, 1e-5
    mg, mo = pair(G, O, order)
    orbs = W.orbitals(2, seed=5)
    tg = []
    for f in orbs:
        t = G.FunctionTree(mg)
        G.project(prec, t, f)
        tg.append(t)
    to = [to_oracle(O, mo, t) for t in tg]
    pg, po = G.FunctionTree(mg), O.FunctionTree(mo)
    for t in tg:
        G.build_grid(pg, t)
    for t in to:
        O.build_grid(po, t)
    G.multiply(-1.0, pg, 1.0, tg[0], tg[1], 0)
    O.multiply(-1.0, po, 1.0, to[0], to[1], 0)
    assert_same_tree(pg.export(), po.export())
    vg, vo = G.FunctionTree(mg), O.FunctionTree(mo)
    G.apply(prec, vg, G.PoissonOperator(mg, prec), pg)
    O.apply(prec, vo, O.PoissonOperator(mo, prec), to_oracle(O, mo, pg))
    assert_same_tree(vg.export(), vo.export())


def test_multiply_errors(gpu_mod):
    G = gpu_mod
    mg = G.MultiResolutionAnalysis(*WORLD, 5, 14)
    a, empty = G.FunctionTree(mg), G.FunctionTree(mg)
    G.project(1e-3, a, gauss(G, A1, C1))
    with pytest.raises(G.MWError):
        G.multiply(1e-3, G.FunctionTree(mg), 1.0, a, empty)  # empty factor
    with pytest.raises(G.MWError):
        G.multiply(1e-3, a, 1.0, a, a)  # output aliases an input
    other = G.MultiResolutionAnalysis(*WORLD, 7, 14)
    b = G.FunctionTree(other)
    G.project(1e-3, b, gauss(G, A2, C2))
    with pytest.raises(G.MWError):
        G.multiply(1e-3, G.FunctionTree(mg), 1.0, a, b)  # different worlds


def test_tree_distance(gpu_mod):
    """||a - b|| from coefficient differences: zero for a tree and itself, equal to the norm identity
    for well-separated trees, symmetric, and exact for a rescaled copy on the same grid"""
    G = gpu_mod
    mg = G.MultiResolutionAnalysis(*WORLD, 5, 14)
    a, b = G.FunctionTree(mg), G.FunctionTree(mg)
    G.project(1e-4, a, gauss(G, A1, C1))
    G.project(1e-4, b, gauss(G, A2, C2))
    assert G.distance(a, a) == 0.0
    d = G.distance(a, b)
    ident = np.sqrt(a.square_norm() + b.square_norm() - 2 * G.dot(a, b))
    assert abs(d - ident) < 1e-10 * ident
    assert abs(G.distance(b, a) - d) < 1e-14 * d
    c = G.FunctionTree(mg)
    G.project(1e-4, c, gauss(G, A1, C1))
    c.rescale(1.0 + 1e-9)
    assert abs(G.distance(a, c) - 1e-9 * np.sqrt(a.square_norm())) < 1e-3 * 1e-9 * np.sqrt(a.square_norm())
