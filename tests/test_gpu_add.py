"""GPU parity of the linear combination (mrcpp::add contract, reference
src/qmfunctions/qmfunction_utils.cpp:170-177) against the FP64 CPU oracle, in the adaptive form and the
union-grid form, and against the projection of the summed function.

Bar: integer tree structure identical; FP64 coefficients within 1e-10 of the largest coefficient.
"""
import numpy as np
import pytest

from test_gpu_parity import WORLD, assert_same_tree, pair, to_oracle

pytestmark = pytest.mark.gpu

TERMS = [(1.0, 2.0, (0.1, -0.2, 0.3)), (-0.5, 30.0, (-0.5, 0.2, 0.1)), (0.25, 8.0, (0.4, 0.4, -0.3))]


def inputs(G, m, prec):
    ts = []
    for _, a, c in TERMS:
        t = G.FunctionTree(m)
        G.project(prec, t, G.gauss_params([1.0], [a], [c]))
        ts.append(t)
    return ts


@pytest.mark.parametrize("order,prec", [(5, 1e-4), (7, 1e-6)])
def test_add_adaptive_parity(gpu_mod, oracle_mod, order, prec):
    G, O = gpu_mod, oracle_mod
    mg, mo = pair(G, O, order)
    tg = inputs(G, mg, prec)
    to = [to_oracle(O, mo, t) for t in tg]
    c = [w for w, _, _ in TERMS]
    sg, so = G.FunctionTree(mg), O.FunctionTree(mo)
    G.add(prec, sg, c, tg)
    O.add(prec, so, c, to)
    assert_same_tree(sg.export(), so.export())
    assert abs(sg.square_norm() - so.square_norm()) < 1e-12 * so.square_norm()


def test_add_union_grid_exact(gpu_mod, oracle_mod):
    """union grid + maxIter 0: the sum is exact, ||sum|| from the inputs' norms and inner products"""
    G, O = gpu_mod, oracle_mod
    mg, mo = pair(G, O, 7)
    tg = inputs(G, mg, 1e-5)
    c = [w for w, _, _ in TERMS]
    sg = G.FunctionTree(mg)
    for t in tg:
        G.build_grid(sg, t)
    G.add(-1.0, sg, c, tg, 0)
    so = O.FunctionTree(mo)
    to = [to_oracle(O, mo, t) for t in tg]
    for t in to:
        O.build_grid(so, t)
    O.add(-1.0, so, c, to, 0)
    assert_same_tree(sg.export(), so.export())
    exact = sum(c[i] * c[j] * G.dot(tg[i], tg[j]) for i in range(3) for j in range(3))
    assert abs(sg.square_norm() - exact) < 1e-12 * exact


def test_add_against_projected_sum(gpu_mod):
    G = gpu_mod
    mg = G.MultiResolutionAnalysis(*WORLD, 7, 14)
    prec = 1e-6
    tg = inputs(G, mg, prec)
    sg = G.FunctionTree(mg)
    G.add(prec, sg, [w for w, _, _ in TERMS], tg)
    eg = G.FunctionTree(mg)
    G.project(prec, eg, G.gauss_params([w for w, _, _ in TERMS], [a for _, a, _ in TERMS], [c for _, _, c in TERMS]))
    assert G.distance(sg, eg) < 20 * prec * np.sqrt(eg.square_norm())


def test_add_errors(gpu_mod):
    G = gpu_mod
    mg = G.MultiResolutionAnalysis(*WORLD, 5, 14)
    t = inputs(G, mg, 1e-3)[0]
    with pytest.raises(G.MWError):
        G.add(1e-3, G.FunctionTree(mg), [], [])
    with pytest.raises(G.MWError):
        G.add(1e-3, t, [1.0], [t])  # output is an input
    with pytest.raises(G.MWError):
        G.add(1e-3, G.FunctionTree(mg), [1.0, 1.0], [t, G.FunctionTree(mg)])  # empty input
    other = G.MultiResolutionAnalysis(*WORLD, 7, 14)
    with pytest.raises(G.MWError):
        G.add(1e-3, G.FunctionTree(other), [1.0], [t])  # different worlds
