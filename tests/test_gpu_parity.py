"""GPU parity: the sm_100a path (through the C-ABI) against the FP64 CPU oracle on the same inputs.

Bar: integer tree structure (node keys) identical; FP64 coefficients within 1e-10 of the largest
coefficient (observed ~1e-13: only summation order differs).  Inputs are projected on the GPU and
loaded unchanged into the oracle, so both sides apply to the identical input tree.
"""
import json
import os

import numpy as np
import pytest
from scipy.special import erf

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
WORLD = (-2, (-5, -5, -5), (10, 10, 10))
COEF_TOL = 1e-10


def keyed(ex):
    return {(int(d), *map(int, t)): i for i, (d, t) in enumerate(zip(ex["depth"], ex["trans"]))}


def assert_same_tree(eg, eo, tol=COEF_TOL):
    kg, ko = keyed(eg), keyed(eo)
    assert set(kg) == set(ko), f"structure differs: {len(kg)} vs {len(ko)} nodes"
    scale = max(np.abs(eo["coef"]).max(), 1e-300)
    diff = max(np.abs(eg["coef"][kg[q]] - eo["coef"][ko[q]]).max() for q in kg)
    assert diff <= tol * scale, (diff, scale)
    # parent / child links describe the same tree
    for q, i in kg.items():
        j = ko[q]
        pg, po = eg["parent"][i], eo["parent"][j]
        if pg < 0:
            assert po < 0
        else:
            assert (int(eg["depth"][pg]), *map(int, eg["trans"][pg])) == (int(eo["depth"][po]), *map(int, eo["trans"][po]))
        assert (eg["child0"][i] < 0) == (eo["child0"][j] < 0)
    return diff / scale


def to_oracle(O, mo, tree_g):
    ex = tree_g.export()
    t = O.FunctionTree(mo)
    t.load(ex["depth"], ex["trans"], ex["parent"], ex["child0"], ex["coef"])
    return t


def pair(G, O, order, max_depth=14, basis=0, world=WORLD):
    return (G.MultiResolutionAnalysis(*world, order, max_depth, basis=basis),
            O.MultiResolutionAnalysis(*world, order, max_depth, basis=basis))


def two_gaussians(G):
    return G.gauss_params([(10 / np.pi) ** 1.5, 0.5 * (30 / np.pi) ** 1.5], [10.0, 30.0],
                          [(0.1, -0.2, 0.3), (-0.5, 0.4, 0.0)])


@pytest.mark.parametrize("order,prec,basis", [(5, 1e-3, 0), (7, 1e-5, 0), (9, 1e-6, 0), (7, 1e-5, 1)])
def test_projection_parity(gpu_mod, oracle_mod, order, prec, basis):
    G, O = gpu_mod, oracle_mod
    mg, mo = pair(G, O, order, basis=basis)
    assert np.abs(mg.filter() - mo.filter()).max() < 1e-10
    f = two_gaussians(G)
    tg = G.FunctionTree(mg)
    G.project(prec, tg, f)
    to = O.FunctionTree(mo)
    O.project(prec, to, f)
    assert_same_tree(tg.export(), to.export())
    assert abs(tg.square_norm() - to.square_norm()) < 1e-12 * to.square_norm()


@pytest.mark.parametrize("order,prec,mu", [(5, 1e-3, 0.0), (5, 1e-3, 1.3), (7, 1e-5, 0.0), (7, 1e-5, 2.0),
                                           (9, 1e-6, 0.0), (9, 1e-6, 0.8)])
def test_apply_parity(gpu_mod, oracle_mod, order, prec, mu):
    G, O = gpu_mod, oracle_mod
    mg, mo = pair(G, O, order)
    inp = G.FunctionTree(mg)
    G.project(prec, inp, two_gaussians(G))
    inp_o = to_oracle(O, mo, inp)
    out = G.FunctionTree(mg)
    sg = G.apply(prec, out, G.ConvolutionOperator(mg, mu, prec), inp)
    out_o = O.FunctionTree(mo)
    so = O.apply(prec, out_o, O.ConvolutionOperator(mo, mu, prec), inp_o)
    assert sg[0] == so[0], "contracted triple counts differ"
    assert sg[2] == so[2], "refinement pass counts differ"
    assert_same_tree(out.export(), out_o.export())
    assert abs(G.dot(out, inp) - O.dot(out_o, inp_o)) < 1e-11 * abs(O.dot(out_o, inp_o))


def test_batched_apply_equals_single_applies(gpu_mod):
    """mw_apply_batched over several trees/operators gives exactly the single-apply results."""
    from mrchem_b200 import workloads as W

    G = gpu_mod
    prec = 1e-5
    m = G.MultiResolutionAnalysis(*WORLD, 7, 14)
    orbs = W.orbitals(5, seed=11)
    mus = W.helmholtz_mus(5, seed=11)
    inps, ops = [], []
    for f, mu in zip(orbs, mus):
        t = G.FunctionTree(m)
        G.project(prec, t, f)
        inps.append(t)
        ops.append(G.HelmholtzOperator(m, mu, prec))
    ops[2] = G.PoissonOperator(m, prec)  # mixed operator kinds in one batch
    outs_b = [G.FunctionTree(m) for _ in inps]
    total = G.apply_batched(prec, outs_b, ops, inps)
    singles = 0
    for i in range(len(inps)):
        o = G.FunctionTree(m)
        singles += G.apply(prec, o, ops[i], inps[i])[0]
        assert_same_tree(outs_b[i].export(), o.export(), tol=0.0)
    assert total == singles


@pytest.mark.parametrize("order,prec,mu", [(7, 1e-5, 0.0), (9, 1e-6, 1.1)])
def test_mixed_precision_apply_error(gpu_mod, order, prec, mu):
    """FP32 products with FP64 accumulation: relative L2 error vs the FP64 apply stays below
    prec / 10 (1e-7 at prec 1e-6); tree structure is the FP64 one up to borderline nodes."""
    G = gpu_mod
    m = G.MultiResolutionAnalysis(*WORLD, order, 14)
    inp = G.FunctionTree(m)
    G.project(prec, inp, two_gaussians(G))
    op = G.ConvolutionOperator(m, mu, prec)
    o64, o32 = G.FunctionTree(m), G.FunctionTree(m)
    G.apply(prec, o64, op, inp, G.APPLY_FP64)
    G.apply(prec, o32, op, inp, G.APPLY_FP32)
    err = G.distance(o32, o64) / np.sqrt(o64.square_norm())
    assert err < 0.1 * prec, err
    assert set(keyed(o32.export(False))) == set(keyed(o64.export(False)))


def test_apply_matches_analytic_potential(gpu_mod, oracle_mod):
    """Poisson of a normalised Gaussian is erf(sqrt(a) r)/r (config-1 accuracy level)."""
    G, O = gpu_mod, oracle_mod
    prec = 1e-5
    mg, mo = pair(G, O, 7)
    alpha, c = 25.0, np.array([0.3, 0.1, -0.2])
    inp = G.FunctionTree(mg)
    G.project(prec, inp, G.gauss_params([(alpha / np.pi) ** 1.5], [alpha], [c]))
    out = G.FunctionTree(mg)
    G.apply(prec, out, G.PoissonOperator(mg, prec), inp)
    ev = to_oracle(O, mo, out)
    rng = np.random.default_rng(3)
    err = 0.0
    for _ in range(300):
        r = c + rng.uniform(-5, 5, 3)
        d = np.linalg.norm(r - c)
        err = max(err, abs(ev.evalf(r) - erf(np.sqrt(alpha) * d) / d))
    assert err < 2e-5 * 2 * np.sqrt(alpha / np.pi)


def test_config1_poisson(gpu_mod, oracle_mod):
    """Config 1 as specified: order 7, prec 1e-5, 3 unit Gaussians (seed 1); parity + analytic."""
    from mrchem_b200 import workloads as W

    G, O = gpu_mod, oracle_mod
    prec = 1e-5
    mg, mo = pair(G, O, 7, max_depth=15)
    f, meta = W.poisson_density(seed=1)
    inp = G.FunctionTree(mg)
    G.project(prec, inp, f)
    out = G.FunctionTree(mg)
    G.apply(prec, out, G.PoissonOperator(mg, prec), inp)
    out_o = O.FunctionTree(mo)
    O.apply(prec, out_o, O.PoissonOperator(mo, prec), to_oracle(O, mo, inp))
    assert_same_tree(out.export(), out_o.export())
    rng = np.random.default_rng(5)
    err, vmax = 0.0, 0.0
    for _ in range(200):
        r = rng.uniform(-6, 6, 3)
        v = sum(erf(np.sqrt(a) * np.linalg.norm(r - c)) / np.linalg.norm(r - c)
                for a, c in zip(meta["alphas"], meta["centers"]))
        err = max(err, abs(out_o.evalf(r) - v))
        vmax = max(vmax, v)
    assert err < 3e-5 * vmax


def test_config2_orbitals_helmholtz_subset(gpu_mod, oracle_mod):
    """Two orbitals of config 2 (order 9, prec 1e-6, Helmholtz mu from the seeded draw)."""
    from mrchem_b200 import workloads as W

    G, O = gpu_mod, oracle_mod
    prec = 1e-6
    mg, mo = pair(G, O, 9, max_depth=15)
    orbs = W.orbitals(32, seed=2)
    mus = W.helmholtz_mus(32, seed=2)
    for i in (0, 7):
        inp = G.FunctionTree(mg)
        G.project(prec, inp, orbs[i])
        assert abs(inp.square_norm() - 1.0) < 1e-5
        out = G.FunctionTree(mg)
        G.apply(prec, out, G.HelmholtzOperator(mg, mus[i], prec), inp)
        out_o = O.FunctionTree(mo)
        O.apply(prec, out_o, O.HelmholtzOperator(mo, mus[i], prec), to_oracle(O, mo, inp))
        assert_same_tree(out.export(), out_o.export())


def test_hydrogen_coulomb_kat(gpu_mod, oracle_mod):
    """Reference KAT quantities (tests/qmoperators/coulomb_operator.cpp) through the GPU path."""
    G = gpu_mod
    kat = json.load(open(os.path.join(HERE, "golden", "reference_kats.json")))
    w = kat["world"]
    m = G.MultiResolutionAnalysis(w["min_scale"], w["corner"], w["boxes"], 7, w["max_depth"])
    orbs = [tuple(o) for o in kat["orbitals"]]
    prec = 1e-5
    rho = G.FunctionTree(m)
    G.project(prec, rho, G.hydrogen_params([(2.0, o, o) for o in orbs]))
    V = G.FunctionTree(m)
    G.apply(prec / np.sqrt(rho.square_norm()), V, G.PoissonOperator(m, prec), rho)
    for key, expr in kat["analytic_E_P"].items():
        i, j = map(int, key.split(","))
        d = G.FunctionTree(m)
        G.project(1e-7, d, G.hydrogen_params([(1.0, orbs[i], orbs[j])]))
        val = G.dot(d, V)
        exact = eval(expr)
        assert abs(val - exact) / exact < 1e-4


@pytest.mark.parametrize("flags", [0, 1, 3])
def test_hydrogen_coulomb_hessian_kat(gpu_mod, flags):
    """tests/qmoperators/coulomb_hessian.cpp:95-98 through the GPU path (FP64, FP32 and BF16x3
    contractions): V = P[rho_1], rho_1 = 4 (1s 2s + 2s 2p1), against the exact integrals the E_P
    quantities converge to (1e-4 at order 9, prec 1e-6), and the reference's own values to 0.5 %."""
    G = gpu_mod
    kat = json.load(open(os.path.join(HERE, "golden", "reference_kats.json")))
    w = kat["world"]
    m = G.MultiResolutionAnalysis(w["min_scale"], w["corner"], w["boxes"], 9, w["max_depth"])
    phi = [tuple(o) for o in kat["hessian"]["phi"]]
    x = [tuple(o) for o in kat["hessian"]["x"]]
    prec = 1e-6
    rho = G.FunctionTree(m)
    G.project(prec, rho, G.hydrogen_params([(4.0, p, q) for p, q in zip(phi, x)]))
    V = G.FunctionTree(m)
    G.apply(prec / np.sqrt(rho.square_norm()), V, G.PoissonOperator(m, prec), rho, flags)
    for key, expr in kat["analytic_hessian_E_P"].items():
        i, j = map(int, key.split(","))
        d = G.FunctionTree(m)
        G.project(1e-7, d, G.hydrogen_params([(1.0, phi[i], phi[j])]))
        val = G.dot(d, V)
        exact = eval(expr)
        assert abs(val - exact) / exact < 1e-4, (key, val, exact)
        ref = kat["coulomb_hessian_E_P"][key]
        assert abs(val - ref) / ref < 5e-3, (key, val, ref)


@pytest.mark.parametrize("flags", [0, 1])
def test_order11_prec1e7_against_oracle(gpu_mod, oracle_mod, flags):
    """Order 11 (k = 12), prec 1e-7 (the finest setting of the precision sweep): FP64 (pencil kernel
    k_bapply<12, double>) and FP32 (k_gapply<12, float>) against the FP64 CPU apply -- identical node
    keys; FP64 coefficients to 1e-10 of the largest, FP32 relative error at most prec (measured 5e-8:
    FP32 products carry about 6e-8 relative rounding, so at prec 1e-7 they use half the budget)."""
    G, O = gpu_mod, oracle_mod
    prec, mu = 1e-7, 1.1
    mg, mo = pair(G, O, 11, max_depth=15)
    inp = G.FunctionTree(mg)
    G.project(prec, inp, two_gaussians(G))
    out = G.FunctionTree(mg)
    G.apply(prec, out, G.HelmholtzOperator(mg, mu, prec), inp, flags)
    out_o = O.FunctionTree(mo)
    O.apply(prec, out_o, O.HelmholtzOperator(mo, mu, prec), to_oracle(O, mo, inp))
    eg, eo = out.export(), out_o.export()
    if flags == 0:
        assert_same_tree(eg, eo)
    else:
        assert set(keyed(eg)) == set(keyed(eo))
        back = G.FunctionTree(mg)
        back.load(eo["depth"], eo["trans"], eo["parent"], eo["child0"], eo["coef"])
        assert G.distance(out, back) / np.sqrt(back.square_norm()) <= prec


@pytest.mark.parametrize("flags", [0, 1, 3])
def test_exchange_pair_against_oracle(gpu_mod, oracle_mod, flags):
    """One exchange pair of the 16-orbital batch at order 9, prec 1e-6 (ExchangePotential.cpp:253,137):
    the MW product phi_0 phi_5 and its Poisson potential against the oracle's -- identical node keys for
    both; the product to 1e-10, the potential to 1e-10 (FP64) or relative error <= 2e-7 (FP32, BF16x3)."""
    from mrchem_b200 import workloads as W

    G, O = gpu_mod, oracle_mod
    prec = 1e-6
    mg, mo = pair(G, O, 9, max_depth=15)
    orbs = W.orbitals(16, seed=2)
    a, b = G.FunctionTree(mg), G.FunctionTree(mg)
    G.project(prec, a, orbs[0])
    G.project(prec, b, orbs[5])
    prod = G.FunctionTree(mg)
    G.multiply(prec, prod, 1.0, a, b)
    prod_o = O.FunctionTree(mo)
    O.multiply(prec, prod_o, 1.0, to_oracle(O, mo, a), to_oracle(O, mo, b))
    assert_same_tree(prod.export(), prod_o.export())
    pot = G.FunctionTree(mg)
    G.apply(prec, pot, G.PoissonOperator(mg, prec), prod, flags)
    pot_o = O.FunctionTree(mo)
    O.apply(prec, pot_o, O.PoissonOperator(mo, prec), to_oracle(O, mo, prod))
    eg, eo = pot.export(), pot_o.export()
    if flags == 0:
        assert_same_tree(eg, eo)
    else:
        assert set(keyed(eg)) == set(keyed(eo))
        back = G.FunctionTree(mg)
        back.load(eo["depth"], eo["trans"], eo["parent"], eo["child0"], eo["coef"])
        assert G.distance(pot, back) / np.sqrt(back.square_norm()) <= 2e-7


def test_config4_density_against_oracle(gpu_mod, oracle_mod):
    """The Poisson potential of the 20-atom density (4 normalised Gaussians per atom, exponents
    log-U[0.3, 1e3]; CoulombPotential.cpp:85) at order 7, prec 1e-5, on the 10^3-root world: FP64,
    FP32 and BF16x3 against the oracle's FP64 apply of the same input tree -- identical node keys for
    every engine; FP64 coefficients to 1e-10 of the largest, the mixed engines' relative error below
    prec / 10 (measured 1e-8 FP32, 4e-8 BF16x3 against the GPU FP64 potential)."""
    from mrchem_b200 import workloads as W

    G, O = gpu_mod, oracle_mod
    prec = 1e-5
    world = (W.WORLD["min_scale"], W.WORLD["corner"], W.WORLD["boxes"])
    mg, mo = pair(G, O, 7, max_depth=15, world=world)
    rho = G.FunctionTree(mg)
    G.project(prec, rho, W.density_20_atoms())
    pot_o = O.FunctionTree(mo)
    O.apply(prec, pot_o, O.PoissonOperator(mo, prec), to_oracle(O, mo, rho))
    eo = pot_o.export()
    back = G.FunctionTree(mg)
    back.load(eo["depth"], eo["trans"], eo["parent"], eo["child0"], eo["coef"])
    P = G.PoissonOperator(mg, prec)
    for flags in (G.APPLY_FP64, G.APPLY_FP32, G.APPLY_BF16X3):
        pot = G.FunctionTree(mg)
        G.apply(prec, pot, P, rho, flags)
        eg = pot.export()
        if flags == G.APPLY_FP64:
            assert_same_tree(eg, eo)
        else:
            assert set(keyed(eg)) == set(keyed(eo)), flags
            assert G.distance(pot, back) / np.sqrt(back.square_norm()) <= prec / 10, flags


def test_upload_download_roundtrip(gpu_mod, oracle_mod):
    G, O = gpu_mod, oracle_mod
    mg, mo = pair(G, O, 7)
    to = O.FunctionTree(mo)
    O.project(1e-4, to, two_gaussians(G))
    eo = to.export()
    tg = G.FunctionTree(mg)
    tg.load(eo["depth"], eo["trans"], eo["parent"], eo["child0"], eo["coef"])
    eg = tg.export()
    assert_same_tree(eg, eo, tol=0.0)
    assert abs(tg.square_norm() - to.square_norm()) < 1e-13 * to.square_norm()


def test_ordered_upload_and_export_into(gpu_mod):
    """A tree in the library's own node order is uploaded without reordering; export_into fills
    caller-owned buffers with exactly what export() returns"""
    G = gpu_mod
    m = G.MultiResolutionAnalysis(*WORLD, 7, 14)
    a = G.FunctionTree(m)
    G.project(1e-5, a, two_gaussians(G))
    ea = a.export()
    b = G.FunctionTree(m)
    b.load(ea["depth"], ea["trans"], ea["parent"], ea["child0"], ea["coef"])
    eb = b.export()
    for key in ("depth", "trans", "parent", "child0", "coef"):
        assert np.array_equal(ea[key], eb[key])
    n = a.nnodes()
    bufs = {"depth": np.zeros(n + 5, np.int32), "parent": np.zeros(n + 5, np.int32), "child0": np.zeros(n + 5, np.int32),
            "trans": np.zeros(3 * (n + 5), np.int64), "coef": np.zeros(ea["coef"].size + 10)}
    assert b.export_into(bufs) == n
    assert np.array_equal(bufs["coef"][:ea["coef"].size], ea["coef"].ravel())
    assert np.array_equal(bufs["trans"][:3 * n], ea["trans"].ravel())
    assert np.array_equal(bufs["child0"][:n], ea["child0"])
    with pytest.raises(G.MWError):
        b.export_into(dict(bufs, coef=np.zeros(5)))


def _sibling_groups_reversed(e):
    """The same tree in another valid node order: roots first, then the sibling groups (8 consecutive
    nodes in the library's order) in reverse order, parent / child indices relinked."""
    n = len(e["depth"])
    nroot = int((e["depth"] == 0).sum())
    order = np.array(list(range(nroot)) + [j for g in reversed(range(nroot, n, 8)) for j in range(g, g + 8)])
    pos = np.empty(n, np.int64)
    pos[order] = np.arange(n)
    par, ch = e["parent"][order], e["child0"][order]
    return dict(depth=e["depth"][order], trans=e["trans"][order], coef=e["coef"][order],
                parent=np.where(par < 0, -1, pos[np.maximum(par, 0)]).astype(np.int32),
                child0=np.where(ch < 0, -1, pos[np.maximum(ch, 0)]).astype(np.int32))


def test_batched_upload_and_download(gpu_mod):
    """load_many / export_many_into (mw_tree_upload_many / mw_tree_download_many) give exactly the trees
    and buffers of one load / export_into per tree, for trees in the library's order and in another valid
    order; a batch with an invalid or repeated tree is refused before anything is copied."""
    G = gpu_mod
    m = G.MultiResolutionAnalysis(*WORLD, 7, 14)
    funcs = [two_gaussians(G), G.gauss_params([1.0], [2.0], [(0.2, 0.0, 0.0)]),
             G.gauss_params([3.0], [40.0], [(-0.3, 0.1, 0.2)])]
    src = []
    for f in funcs:
        t = G.FunctionTree(m)
        G.project(1e-5, t, f)
        src.append(t.export())
    arrays = [src[0], _sibling_groups_reversed(src[1]), src[2]]
    assert len(src[1]["depth"]) > 1000 and not np.array_equal(arrays[1]["trans"], src[1]["trans"])
    names = ("depth", "trans", "parent", "child0", "coef")
    one = [G.FunctionTree(m) for _ in arrays]
    for t, a in zip(one, arrays):
        t.load(*(a[k] for k in ("depth", "trans", "parent", "child0", "coef")))
    many = [G.FunctionTree(m) for _ in arrays]
    G.load_many(many, arrays)
    for a, b in zip(one, many):
        ea, eb = a.export(), b.export()
        for k in names:
            assert np.array_equal(ea[k], eb[k]), k
        assert a.square_norm() == b.square_norm()
    bufs = []
    for t in many:
        n, k = t.nnodes(), t.mra.k
        bufs.append({"depth": np.zeros(n + 3, np.int32), "parent": np.zeros(n + 3, np.int32),
                     "child0": np.zeros(n + 3, np.int32), "trans": np.zeros(3 * (n + 3), np.int64),
                     "coef": np.zeros(n * (2 * k) ** 3 + 7)})
    counts = G.export_many_into(many, bufs)
    for t, b, c in zip(many, bufs, counts):
        e = t.export()
        assert c == t.nnodes()
        assert np.array_equal(b["depth"][:c], e["depth"])
        assert np.array_equal(b["trans"][:3 * c], e["trans"].ravel())
        assert np.array_equal(b["parent"][:c], e["parent"])
        assert np.array_equal(b["child0"][:c], e["child0"])
        assert np.array_equal(b["coef"][:e["coef"].size], e["coef"].ravel())
    bad = dict(src[1], trans=src[1]["trans"].copy())
    bad["trans"][-1, 0] = 1 << 40
    with pytest.raises(G.MWError):
        G.load_many([many[0], many[1]], [src[2], bad])
    with pytest.raises(G.MWError):
        G.load_many([many[0], many[0]], [src[2], src[2]])
    e0 = many[0].export()
    assert np.array_equal(e0["coef"], src[0]["coef"]) and np.array_equal(e0["trans"], src[0]["trans"])


def test_rescale_and_dot(gpu_mod, oracle_mod):
    G, O = gpu_mod, oracle_mod
    mg, mo = pair(G, O, 5)
    a = G.FunctionTree(mg)
    G.project(1e-3, a, two_gaussians(G))
    b = G.FunctionTree(mg)
    G.project(1e-3, b, G.gauss_params([1.0], [2.0], [(0.2, 0.0, 0.0)]))
    d0 = G.dot(a, b)
    assert abs(d0 - O.dot(to_oracle(O, mo, a), to_oracle(O, mo, b))) < 1e-12 * abs(d0)
    n0 = a.square_norm()
    a.rescale(-1.0 / (2 * np.pi))  # HelmholtzVector.cpp:81
    assert abs(a.square_norm() - n0 / (4 * np.pi ** 2)) < 1e-12 * n0
    assert abs(G.dot(a, b) + d0 / (2 * np.pi)) < 1e-12 * abs(d0)


def test_zero_function(gpu_mod):
    G = gpu_mod
    m = G.MultiResolutionAnalysis(*WORLD, 5, 10)
    z = G.FunctionTree(m)
    G.project(1e-3, z, G.gauss_params([0.0], [1.0], [(0.0, 0.0, 0.0)]))
    assert z.nnodes() == 1000 and z.square_norm() == 0.0
    out = G.FunctionTree(m)
    G.apply(1e-3, out, G.PoissonOperator(m, 1e-3), z)
    assert out.nnodes() == 1000 and out.square_norm() == 0.0


def test_depth_limit(gpu_mod, oracle_mod):
    G, O = gpu_mod, oracle_mod
    mg, mo = pair(G, O, 5, max_depth=2)
    f = G.gauss_params([(200 / np.pi) ** 1.5], [200.0], [(0.05, 0.05, 0.05)])
    tg = G.FunctionTree(mg)
    G.project(1e-6, tg, f)
    assert tg.export()["depth"].max() == 2
    to = O.FunctionTree(mo)
    O.project(1e-6, to, f)
    assert_same_tree(tg.export(), to.export())
    out = G.FunctionTree(mg)
    G.apply(1e-6, out, G.PoissonOperator(mg, 1e-6), tg)
    out_o = O.FunctionTree(mo)
    O.apply(1e-6, out_o, O.PoissonOperator(mo, 1e-6), to_oracle(O, mo, tg))
    assert_same_tree(out.export(), out_o.export())


def test_single_root_world(gpu_mod, oracle_mod):
    G, O = gpu_mod, oracle_mod
    world = (0, (-1, -1, -1), (1, 1, 1))  # one root box [-1, 0)^3 ... edge 1
    mg, mo = pair(G, O, 5, max_depth=8, world=world)
    f = G.gauss_params([1.0], [20.0], [(-0.5, -0.5, -0.5)])
    tg = G.FunctionTree(mg)
    G.project(1e-4, tg, f)
    out = G.FunctionTree(mg)
    G.apply(1e-4, out, G.HelmholtzOperator(mg, 1.0, 1e-4), tg)
    out_o = O.FunctionTree(mo)
    O.apply(1e-4, out_o, O.HelmholtzOperator(mo, 1.0, 1e-4), to_oracle(O, mo, tg))
    assert_same_tree(out.export(), out_o.export())


def test_errors_are_reported(gpu_mod):
    G = gpu_mod
    with pytest.raises(G.MWError):
        G.MultiResolutionAnalysis(*WORLD, 15, 10)  # order out of range
    m1 = G.MultiResolutionAnalysis(*WORLD, 5, 10)
    m2 = G.MultiResolutionAnalysis(*WORLD, 5, 10)
    a = G.FunctionTree(m1)
    G.project(1e-3, a, G.gauss_params([1.0], [1.0], [(0.0, 0.0, 0.0)]))
    with pytest.raises(G.MWError):
        G.apply(1e-3, G.FunctionTree(m2), G.PoissonOperator(m1, 1e-3), a)  # different worlds
    with pytest.raises(G.MWError):
        G.apply(1e-3, G.FunctionTree(m1), G.PoissonOperator(m1, 1e-3), G.FunctionTree(m1))  # empty input
    with pytest.raises(G.MWError):
        G.HelmholtzOperator(m1, -1.0, 1e-3)
    with pytest.raises(G.MWError):
        G.project(1e-3, a, (7, np.array([1.0])))  # unknown function type
    # the context still works after the errors
    b = G.FunctionTree(m1)
    G.project(1e-3, b, G.gauss_params([1.0], [1.0], [(0.0, 0.0, 0.0)]))
    assert b.square_norm() > 0
