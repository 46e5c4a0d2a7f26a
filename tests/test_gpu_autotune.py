"""Contraction work split per engine (mw_ctx_set_chunk_triples) and its autotuner on the GPU: every
chunk size gives the same tree and coefficients up to FP64 rounding (only the grouping of partial
sums changes), invalid values are rejected, and the tuner leaves a measured candidate set."""
import numpy as np
import pytest

from test_gpu_parity import WORLD, two_gaussians

pytestmark = pytest.mark.gpu


def test_chunk_sizes_agree_and_tuner_sets_one(gpu_mod):
    from mrchem_b200.autotune import tune_chunk_triples

    G = gpu_mod
    ctx = G.Context(0)
    m = G.MultiResolutionAnalysis(*WORLD, 7, 14, ctx=ctx)
    inp = G.FunctionTree(m)
    G.project(1e-5, inp, two_gaussians(G))
    op = G.PoissonOperator(m, 1e-5)
    assert ctx.chunk_triples(G.APPLY_FP64) == 48
    ref = None
    for flags in (G.APPLY_FP64, G.APPLY_FP32):
        outs = {}
        for c in (1, 7, 48, 4096):
            ctx.set_chunk_triples(flags, c)
            o = G.FunctionTree(m)
            G.apply(1e-5, o, op, inp, flags)
            outs[c] = o
        for c, o in outs.items():
            assert o.nnodes() == outs[48].nnodes()
            assert G.distance(o, outs[48]) <= 1e-12 * np.sqrt(outs[48].square_norm()), (flags, c)
        if flags == G.APPLY_FP64:
            ref = outs[48]
    with pytest.raises(G.MWError):
        ctx.set_chunk_triples(G.APPLY_FP32, 0)
    with pytest.raises(G.MWError):
        ctx.set_chunk_triples(7, 48)
    o = G.FunctionTree(m)
    res = tune_chunk_triples(ctx, lambda: G.apply(1e-5, o, op, inp, G.APPLY_FP64), G.APPLY_FP64,
                             candidates=(16, 48, 128), reps=1, warmup=1)
    assert res["best"] in (16, 48, 128) and ctx.chunk_triples(G.APPLY_FP64) == res["best"]
    assert G.distance(o, ref) <= 1e-12 * np.sqrt(ref.square_norm())
