"""Handle lifetimes through the C-ABI: a context or world may be destroyed while trees, operators or
networks still point to it (e.g. by a garbage collector finalising a reference cycle in any order);
it is freed with the last of them.  Destroying a handle twice is an error, not a crash."""
import gc

import pytest

from test_gpu_parity import WORLD, two_gaussians

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ctx_first", [True, False])
def test_parents_destroyed_first(gpu_mod, ctx_first):
    G = gpu_mod
    L = G.load_library()
    ctx = G.Context(0)
    m = G.MultiResolutionAnalysis(*WORLD, 5, 12, ctx=ctx)
    t = G.FunctionTree(m)
    G.project(1e-3, t, two_gaussians(G))
    op = G.PoissonOperator(m, 1e-3)
    out = G.FunctionTree(m)
    G.apply(1e-3, out, op, t)
    n_before, norm_before = out.nnodes(), out.square_norm()
    net = G.ProposalNet(ctx=ctx, hidden_layers=1, width=16, seed=1)
    if ctx_first:
        assert L.mw_ctx_destroy(ctx._h) == 0
        ctx._h = None
    assert L.mw_mra_destroy(m._h) == 0
    m._h = None
    # the children still work: the world (and context) stay alive until the last one goes
    assert out.nnodes() == n_before
    assert out.square_norm() == norm_before
    for h in (t, out):
        assert L.mw_tree_destroy(h._h) == 0
        h._h = None
    assert L.mw_op_destroy(op._h) == 0
    op._h = None
    assert L.mw_mlp_destroy(net._h) == 0
    net._h = None
    if not ctx_first:
        assert L.mw_ctx_destroy(ctx._h) == 0
        ctx._h = None


def test_double_destroy_is_an_error(gpu_mod):
    G = gpu_mod
    L = G.load_library()
    ctx = G.Context(0)
    m = G.MultiResolutionAnalysis(*WORLD, 5, 12, ctx=ctx)
    t = G.FunctionTree(m)
    assert L.mw_mra_destroy(m._h) == 0
    assert L.mw_mra_destroy(m._h) == -1  # MW_ERR_ARG: the world is closed, still held by the tree
    m._h = None
    assert L.mw_tree_destroy(t._h) == 0  # frees the world
    t._h = None


def test_reference_cycle_collected_in_any_order(gpu_mod):
    """Objects in one garbage cycle are finalised in arbitrary order."""
    G = gpu_mod
    for _ in range(3):
        m = G.MultiResolutionAnalysis(*WORLD, 5, 12)
        t = G.FunctionTree(m)
        G.project(1e-3, t, two_gaussians(G))
        box = {"m": m, "t": t}
        box["self"] = box
        m._cycle = box
        del m, t, box
        gc.collect()
