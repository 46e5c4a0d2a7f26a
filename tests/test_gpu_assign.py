"""mw_tree_assign: a deep device-to-device copy of a tree, also between contexts (streams) of one device
on worlds with the same parameters, bit for bit; the copy works as an apply input in its own context.
Mismatched worlds and self-assignment are rejected."""
import numpy as np
import pytest

from test_gpu_parity import WORLD, two_gaussians

pytestmark = pytest.mark.gpu


def test_assign_across_contexts(gpu_mod):
    G = gpu_mod
    ca, cb = G.Context(0), G.Context(0)
    ma = G.MultiResolutionAnalysis(*WORLD, 7, 14, ctx=ca)
    mb = G.MultiResolutionAnalysis(*WORLD, 7, 14, ctx=cb)
    src = G.FunctionTree(mb)
    G.project(1e-5, src, two_gaussians(G))
    dst = G.FunctionTree(ma)
    G.project(1e-3, dst, two_gaussians(G))  # non-empty: replaced
    dst.assign(src)
    ea, eb = dst.export(), src.export()
    for key in ("depth", "trans", "parent", "child0", "coef"):
        assert np.array_equal(ea[key], eb[key]), key
    assert dst.square_norm() == src.square_norm()
    # the copy is an input of an apply in its own context, with the same result as the original's
    P_a, P_b = G.PoissonOperator(ma, 1e-5), G.PoissonOperator(mb, 1e-5)
    oa, ob = G.FunctionTree(ma), G.FunctionTree(mb)
    G.apply(1e-5, oa, P_a, dst)
    G.apply(1e-5, ob, P_b, src)
    xa, xb = oa.export(), ob.export()
    assert np.array_equal(xa["coef"], xb["coef"]) and np.array_equal(xa["depth"], xb["depth"])
    # and back into the other context
    back = G.FunctionTree(mb)
    back.assign(oa)
    assert np.array_equal(back.export()["coef"], xb["coef"])


def test_assign_rejects_mismatch(gpu_mod):
    G = gpu_mod
    m7 = G.MultiResolutionAnalysis(*WORLD, 7, 14)
    m5 = G.MultiResolutionAnalysis(*WORLD, 5, 14)
    t7 = G.FunctionTree(m7)
    G.project(1e-3, t7, two_gaussians(G))
    with pytest.raises(G.MWError):
        G.FunctionTree(m5).assign(t7)
    with pytest.raises(G.MWError):
        t7.assign(t7)
