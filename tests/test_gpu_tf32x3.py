"""GPU tests of the tensor-core contraction (flag MW_APPLY_TF32X3: tcgen05 split-TF32 products with the
data in two TF32 pieces and the operators in three, FP32 sums inside a term, compensated summation over
terms).

Bars: relative L2 error against the FP64 apply, and against the FP64 CPU oracle, below the requested
precision `prec` (the FP32 CUDA-core path stays below prec / 10; the two-piece data split carries about
22 of FP32's 24 bits, and the tensor core's FP32 accumulation truncates); node keys identical to the
FP64 tree and to the oracle's (refinement decisions are FP64 on the computed norms); batched results
bit-identical to single applies (the contraction is deterministic).
"""
import numpy as np
import pytest

from test_gpu_parity import WORLD, keyed, pair, to_oracle, two_gaussians

pytestmark = pytest.mark.gpu


def rel_err(G, a, b):
    return G.distance(a, b) / np.sqrt(b.square_norm())


@pytest.mark.parametrize("order,prec,mu", [(4, 1e-3, 0.0), (5, 1e-4, 0.5), (7, 1e-5, 0.0), (8, 1e-5, 1.1),
                                           (9, 1e-6, 0.0), (9, 1e-6, 1.1)])
def test_tf32x3_apply_error(gpu_mod, order, prec, mu):
    G = gpu_mod
    m = G.MultiResolutionAnalysis(*WORLD, order, 14)
    inp = G.FunctionTree(m)
    G.project(prec, inp, two_gaussians(G))
    op = G.ConvolutionOperator(m, mu, prec)
    o64, otc = G.FunctionTree(m), G.FunctionTree(m)
    G.apply(prec, o64, op, inp, G.APPLY_FP64)
    G.apply(prec, otc, op, inp, G.APPLY_TF32X3)
    err = rel_err(G, otc, o64)
    assert err < prec, err
    assert set(keyed(otc.export(False))) == set(keyed(o64.export(False)))


def test_tf32x3_against_oracle_config2_orbital(gpu_mod, oracle_mod):
    """One orbital of the 32-orbital Helmholtz batch (order 9, prec 1e-6) against the FP64 CPU apply."""
    from mrchem_b200 import workloads as W

    G, O = gpu_mod, oracle_mod
    prec = 1e-6
    mg, mo = pair(G, O, 9, max_depth=15)
    orbs = W.orbitals(32, seed=2)
    mus = W.helmholtz_mus(32, seed=2)
    inp = G.FunctionTree(mg)
    G.project(prec, inp, orbs[3])
    out = G.FunctionTree(mg)
    G.apply(prec, out, G.HelmholtzOperator(mg, mus[3], prec), inp, G.APPLY_TF32X3)
    out_o = O.FunctionTree(mo)
    O.apply(prec, out_o, O.HelmholtzOperator(mo, mus[3], prec), to_oracle(O, mo, inp))
    back = G.FunctionTree(mg)
    ex = out_o.export()
    back.load(ex["depth"], ex["trans"], ex["parent"], ex["child0"], ex["coef"])
    err = rel_err(G, out, back)
    assert err < prec, err
    assert set(keyed(out.export(False))) == set(keyed(back.export(False)))


def test_tf32x3_batched_equals_single(gpu_mod):
    from mrchem_b200 import workloads as W

    G = gpu_mod
    prec = 1e-6
    m = G.MultiResolutionAnalysis(*WORLD, 9, 15)
    orbs = W.orbitals(3, seed=5)
    mus = W.helmholtz_mus(3, seed=5)
    inps, ops = [], []
    for f, mu in zip(orbs, mus):
        t = G.FunctionTree(m)
        G.project(prec, t, f)
        inps.append(t)
        ops.append(G.HelmholtzOperator(m, mu, prec))
    outs = [G.FunctionTree(m) for _ in inps]
    G.apply_batched(prec, outs, ops, inps, G.APPLY_TF32X3)
    for i in range(len(inps)):
        o = G.FunctionTree(m)
        G.apply(prec, o, ops[i], inps[i], G.APPLY_TF32X3)
        assert o.nnodes() == outs[i].nnodes()
        assert G.distance(o, outs[i]) == 0.0


def test_tf32x3_derivative_and_large_order(gpu_mod):
    """The fixed-grid derivative through the tensor-core contraction (the differentiation cancels
    large terms, which amplifies the data split's rounding: bar 5e-6); order 11 (k = 12, outside the
    tensor-core shared-memory plan) takes the FP32 path under the same flag."""
    G = gpu_mod
    m = G.MultiResolutionAnalysis(*WORLD, 9, 14)
    f = G.FunctionTree(m)
    G.project(1e-6, f, two_gaussians(G))
    D = G.ABGVOperator(m, 0.0, 0.0)
    for d in range(3):
        g64, gtc = G.FunctionTree(m), G.FunctionTree(m)
        G.apply_derivative(g64, D, f, d)
        G.apply_derivative(gtc, D, f, d, G.APPLY_TF32X3)
        assert rel_err(G, gtc, g64) < 5e-6
    m11 = G.MultiResolutionAnalysis(*WORLD, 11, 14)
    inp = G.FunctionTree(m11)
    G.project(1e-5, inp, two_gaussians(G))
    op = G.PoissonOperator(m11, 1e-5)
    o64, otc = G.FunctionTree(m11), G.FunctionTree(m11)
    G.apply(1e-5, o64, op, inp)
    G.apply(1e-5, otc, op, inp, G.APPLY_TF32X3)
    assert rel_err(G, otc, o64) < 1e-6


def test_tf32x3_unknown_flag_rejected(gpu_mod):
    G = gpu_mod
    m = G.MultiResolutionAnalysis(*WORLD, 5, 14)
    inp = G.FunctionTree(m)
    G.project(1e-3, inp, two_gaussians(G))
    with pytest.raises(G.MWError):
        G.apply(1e-3, G.FunctionTree(m), G.PoissonOperator(m, 1e-3), inp, 4)


def test_tf32x3_fine_precision_takes_fp32_engine(gpu_mod):
    """Below prec 1e-6 the split-TF32 error floor (about 2e-7) would exceed the request: the flag runs
    the FP32 engine there, bit for bit."""
    G = gpu_mod
    prec = 1e-7
    m = G.MultiResolutionAnalysis(*WORLD, 7, 14)
    inp = G.FunctionTree(m)
    G.project(prec, inp, two_gaussians(G))
    op = G.PoissonOperator(m, prec)
    o32, otc = G.FunctionTree(m), G.FunctionTree(m)
    G.apply(prec, o32, op, inp, G.APPLY_FP32)
    G.apply(prec, otc, op, inp, G.APPLY_TF32X3)
    assert otc.nnodes() == o32.nnodes()
    assert G.distance(otc, o32) == 0.0
