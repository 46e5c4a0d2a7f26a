"""GPU tests of the BF16x3 contraction engine (flag MW_APPLY_BF16X3): the x mode product of every
(output, input, term) triple on the tcgen05 tensor cores, with data rows written as four and operator
rows as three BF16 slices of a per-row fixed-point form so that the tensor core sums each slice pair
exactly, the y and z
mode products as FP32 products on the CUDA cores, and every term's contribution accumulated in FP64.

Bars: integer tree structure (node keys) identical to the FP64 apply and to the FP64 CPU oracle;
relative L2 error of the coefficients at most prec / 10 (the bar of the FP32 CUDA-core engine);
contracted triple counts equal to the FP64 path's; batched results bit-identical to single applies.
"""
import numpy as np
import pytest

from test_gpu_parity import WORLD, keyed, pair, to_oracle, two_gaussians

pytestmark = pytest.mark.gpu


def rel_err(G, a, b):
    return G.distance(a, b) / np.sqrt(b.square_norm())


def same_keys(G, a, b):
    return set(keyed(a.export(with_coefs=False))) == set(keyed(b.export(with_coefs=False)))


@pytest.mark.parametrize("order,prec,mu", [(6, 1e-5, 0.0), (7, 1e-5, 0.0), (7, 1e-5, 1.1), (8, 1e-6, 0.7),
                                           (9, 1e-6, 0.0), (9, 1e-6, 1.1)])
def test_bf16x3_matches_fp64_apply(gpu_mod, order, prec, mu):
    G = gpu_mod
    m = G.MultiResolutionAnalysis(*WORLD, order, 14)
    inp = G.FunctionTree(m)
    G.project(prec, inp, two_gaussians(G))
    op = G.ConvolutionOperator(m, mu, prec)
    o64, obf = G.FunctionTree(m), G.FunctionTree(m)
    n64 = G.apply(prec, o64, op, inp, G.APPLY_FP64)
    nbf = G.apply(prec, obf, op, inp, G.APPLY_BF16X3)
    err = rel_err(G, obf, o64)
    assert err <= 0.1 * prec, err
    assert same_keys(G, obf, o64)
    assert nbf[0] == n64[0]


@pytest.mark.parametrize("idx", [0, 3, 17])
def test_bf16x3_against_oracle_config2_orbitals(gpu_mod, oracle_mod, idx):
    """Orbitals of the 32-orbital Helmholtz batch (order 9, prec 1e-6) against the FP64 CPU apply:
    identical node keys, relative error at most 2e-7 (prec / 5) and within 2x of the FP32 CUDA-core
    engine's error on the same orbital."""
    from mrchem_b200 import workloads as W

    G, O = gpu_mod, oracle_mod
    prec = 1e-6
    mg, mo = pair(G, O, 9, max_depth=15)
    orbs = W.orbitals(32, seed=2)
    mus = W.helmholtz_mus(32, seed=2)
    inp = G.FunctionTree(mg)
    G.project(prec, inp, orbs[idx])
    out = G.FunctionTree(mg)
    G.apply(prec, out, G.HelmholtzOperator(mg, mus[idx], prec), inp, G.APPLY_BF16X3)
    out_o = O.FunctionTree(mo)
    O.apply(prec, out_o, O.HelmholtzOperator(mo, mus[idx], prec), to_oracle(O, mo, inp))
    back = G.FunctionTree(mg)
    ex = out_o.export()
    back.load(ex["depth"], ex["trans"], ex["parent"], ex["child0"], ex["coef"])
    assert same_keys(G, out, back)
    err = rel_err(G, out, back)
    o32 = G.FunctionTree(mg)
    G.apply(prec, o32, G.HelmholtzOperator(mg, mus[idx], prec), inp, G.APPLY_FP32)
    assert same_keys(G, o32, back)
    err32 = rel_err(G, o32, back)
    assert err <= 2e-7, (err, err32)
    assert err <= 2.0 * err32 + 1e-8, (err, err32)


def test_bf16x3_batched_equals_single(gpu_mod):
    from mrchem_b200 import workloads as W

    G = gpu_mod
    prec = 1e-6
    m = G.MultiResolutionAnalysis(*WORLD, 9, 15)
    orbs = W.orbitals(4, seed=5)
    mus = W.helmholtz_mus(4, seed=5)
    inps, ops = [], []
    for f, mu in zip(orbs, mus):
        t = G.FunctionTree(m)
        G.project(prec, t, f)
        inps.append(t)
        ops.append(G.HelmholtzOperator(m, mu, prec))
    outs = [G.FunctionTree(m) for _ in inps]
    G.apply_batched(prec, outs, ops, inps, G.APPLY_BF16X3)
    for i in range(len(inps)):
        o = G.FunctionTree(m)
        G.apply(prec, o, ops[i], inps[i], G.APPLY_BF16X3)
        assert G.distance(o, outs[i]) == 0.0
        assert same_keys(G, o, outs[i])


def test_bf16x3_unsupported_order_takes_fp32_engine(gpu_mod):
    """Orders outside k = 7..10 run the FP32 engine under the flag: the same result bit for bit."""
    G = gpu_mod
    prec = 1e-4
    m = G.MultiResolutionAnalysis(*WORLD, 4, 12)
    inp = G.FunctionTree(m)
    G.project(prec, inp, two_gaussians(G))
    op = G.PoissonOperator(m, prec)
    a, b = G.FunctionTree(m), G.FunctionTree(m)
    G.apply(prec, a, op, inp, G.APPLY_FP32)
    G.apply(prec, b, op, inp, G.APPLY_BF16X3)
    assert G.distance(a, b) == 0.0


def test_bf16x3_zero_input(gpu_mod):
    G = gpu_mod
    m = G.MultiResolutionAnalysis(*WORLD, 9, 12)
    inp = G.FunctionTree(m)
    G.project(1e-6, inp, G.gauss_params([0.0], [1.0], [(0.0, 0.0, 0.0)]))
    out = G.FunctionTree(m)
    G.apply(1e-6, out, G.PoissonOperator(m, 1e-6), inp, G.APPLY_BF16X3)
    assert out.square_norm() == 0.0
