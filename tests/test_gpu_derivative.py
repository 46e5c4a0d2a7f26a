"""GPU parity of the first-derivative operator (mrcpp::ABGVOperator + apply(out, D, inp, dir) contract,
reference src/SCFDriver.cpp:282-283, src/qmoperators/one_electron/NablaOperator.cpp:35) against the
FP64 CPU oracle, and against the analytic derivative of a Gaussian.

Bar: the output has the input's grid; FP64 coefficients within 1e-10 of the largest coefficient.
"""
import numpy as np
import pytest

from test_gpu_parity import WORLD, assert_same_tree, pair, to_oracle

pytestmark = pytest.mark.gpu

ALPHA, C = 3.0, (0.1, -0.2, 0.3)


@pytest.mark.parametrize("order,ab", [(5, (0.0, 0.0)), (5, (0.5, 0.5)), (7, (0.5, 0.5)), (7, (0.0, 1.0))])
def test_derivative_parity(gpu_mod, oracle_mod, order, ab):
    G, O = gpu_mod, oracle_mod
    mg, mo = pair(G, O, order)
    f = G.FunctionTree(mg)
    G.project(1e-5, f, G.gauss_params([1.0, 0.5], [ALPHA, 20.0], [C, (-0.4, 0.3, 0.0)]))
    fo = to_oracle(O, mo, f)
    D = G.ABGVOperator(mg, *ab)
    for d in range(3):
        g = G.FunctionTree(mg)
        G.apply_derivative(g, D, f, d)
        go = O.FunctionTree(mo)
        O.derivative(go, fo, ab[0], ab[1], d)
        assert g.nnodes() == f.nnodes()
        assert_same_tree(g.export(), go.export())


def test_derivative_analytic_and_mixed(gpu_mod):
    G = gpu_mod
    m = G.MultiResolutionAnalysis(*WORLD, 7, 14)
    prec = 1e-6
    f = G.FunctionTree(m)
    G.project(prec, f, G.gauss_params([1.0], [ALPHA], [C]))
    D = G.ABGVOperator(m, 0.0, 0.0)
    for d in range(3):
        g = G.FunctionTree(m)
        G.apply_derivative(g, D, f, d)
        pw = [0, 0, 0]
        pw[d] = 1
        e = G.FunctionTree(m)
        G.project(prec, e, G.gauss_params([-2 * ALPHA], [ALPHA], [C], [tuple(pw)]))
        assert G.distance(g, e) < 20 * prec * np.sqrt(e.square_norm())
        g32 = G.FunctionTree(m)
        G.apply_derivative(g32, D, f, d, G.APPLY_FP32)
        assert G.distance(g32, g) < 1e-6 * np.sqrt(g.square_norm())


def test_derivative_errors(gpu_mod):
    G = gpu_mod
    m = G.MultiResolutionAnalysis(*WORLD, 5, 14)
    f = G.FunctionTree(m)
    G.project(1e-3, f, G.gauss_params([1.0], [ALPHA], [C]))
    D = G.ABGVOperator(m, 0.5, 0.5)
    with pytest.raises(G.MWError):
        G.apply_derivative(G.FunctionTree(m), D, f, 3)
    with pytest.raises(G.MWError):
        G.apply_derivative(f, D, f, 0)
    with pytest.raises(G.MWError):
        G.ABGVOperator(m, 1.5, 0.0)
    with pytest.raises(G.MWError):  # a derivative is not applied as a convolution
        G.apply(1e-3, G.FunctionTree(m), D, f)
