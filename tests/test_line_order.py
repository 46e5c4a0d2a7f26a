"""The line order of the GEMM-tiled contraction, checked on the CPU (no GPU needed).

The contraction kernel (mrchem_b200/csrc/mw_apply.cu, k_gapply) sorts an output node's surviving
(input node, term) triples by (term, dz, dy) and uses the separability of every Gaussian term,

    sum_l  beta Mz(dz) My(dy) Mx(dx) in_l  =  sum_dz beta Mz(dz) [ sum_dy My(dy) [ sum_dx Mx(dx) in_l ] ],

so that a line (equal term, dz, dy) shares one y mode product and a plane (equal term, dz) one z
mode product.  These tests restate that grouping in numpy with the oracle's own NS-form operator
matrices and compare it with the per-triple sum of the oracle's method, check the oracle's line
statistics of a real apply, and compare whole oracle applies summed in either order.
"""
import numpy as np
import pytest

WORLD = (-2, (-5, -5, -5), (10, 10, 10))


def mode(M, X, d):
    """Mode product along dimension d of a block stored [z][y][x] (x fastest, as the library)."""
    if d == 0:
        return np.einsum("ij,cbj->cbi", M, X)
    if d == 1:
        return np.einsum("ij,cja->cia", M, X)
    return np.einsum("ij,jba->iba", M, X)


def triples_of(op, depth, nterms, band, rng):
    """(term, (dx, dy, dz)) triples in candidate order (offsets outer, terms inner, as the kernel's
    input list) with random input blocks per offset."""
    K2 = 2 * op.mra.k
    offs = [(dx, dy, dz) for dz in range(-band, band + 1) for dy in range(-band, band + 1)
            for dx in range(-band, band + 1)]
    rng.shuffle(offs)
    blocks = {o: rng.standard_normal((K2, K2, K2)) for o in offs}
    terms = []
    for m in range(nterms):
        if all(op.ns_matrix(depth, m, l) is not None for l in range(-band, band + 1)):
            terms.append(m)
    assert len(terms) >= 3
    trip = [(m, o) for o in offs for m in terms]
    return trip, blocks


def test_line_grouping_equals_per_triple_sum(oracle_mod):
    O = oracle_mod
    rng = np.random.default_rng(7)
    m = O.MultiResolutionAnalysis(*WORLD, 5, 10)
    op = O.HelmholtzOperator(m, 1.3, 1e-5)
    alpha, beta = op.terms()
    depth = 2
    trip, blocks = triples_of(op, depth, len(alpha), 1, rng)
    mats = {}

    def M(mi, l):
        if (mi, l) not in mats:
            mats[(mi, l)] = op.ns_matrix(depth, mi, l)
        return mats[(mi, l)]

    # per-triple order of the oracle: three mode products per triple
    ref = sum(beta[mi] * mode(M(mi, dz), mode(M(mi, dy), mode(M(mi, dx), blocks[(dx, dy, dz)], 0), 1), 2)
              for mi, (dx, dy, dz) in trip)
    # line order: a stable sort by (term, dz, dy) of the candidate-ordered triples, then the sums of
    # a line's x products, of a plane's y products and one z product per plane
    order = sorted(range(len(trip)), key=lambda i: (trip[i][0], trip[i][1][2], trip[i][1][1]))
    out = np.zeros_like(ref)
    lines = planes = 0
    t = 0
    while t < len(order):
        mi, (_, _, dz) = trip[order[t]]
        t2 = None
        while t < len(order) and trip[order[t]][0] == mi and trip[order[t]][1][2] == dz:
            dy = trip[order[t]][1][1]
            t1 = None
            while (t < len(order) and trip[order[t]][0] == mi and trip[order[t]][1][2] == dz
                   and trip[order[t]][1][1] == dy):
                dx = trip[order[t]][1][0]
                x = mode(M(mi, dx), blocks[(dx, dy, dz)], 0)
                t1 = x if t1 is None else t1 + x
                t += 1
            y = mode(M(mi, dy), t1, 1)
            t2 = y if t2 is None else t2 + y
            lines += 1
        out += beta[mi] * mode(M(mi, dz), t2, 2)
        planes += 1
    assert np.max(np.abs(out - ref)) <= 1e-12 * np.max(np.abs(ref))
    # a full 3 x 3 x 3 band: 27 triples, 9 lines, 3 planes per term
    nt = len(trip) // 27
    assert (lines, planes) == (9 * nt, 3 * nt)
    assert 3 * len(trip) / (len(trip) + lines + planes) == pytest.approx(81 / 39)


def test_oracle_line_statistics(oracle_mod):
    """On a projected Gaussian sum the oracle reports fewer lines than triples and fewer planes than
    lines; the mode products per triple of the line order, (triples + lines + planes) / triples, lie
    between 1 and 3."""
    O = oracle_mod
    m = O.MultiResolutionAnalysis(*WORLD, 5, 10)
    f = O.FunctionTree(m)
    O.project(1e-4, f, O.gauss_params([1.0, 0.5], [3.0, 20.0], [(0.1, -0.2, 0.3), (-0.4, 0.2, 0.0)]))
    op = O.HelmholtzOperator(m, 1.0, 1e-4)
    g = O.FunctionTree(m)
    triples, lines, planes = O.apply_line_stats(1e-4, g, op, f)
    assert 0 < planes < lines < triples
    per_triple = (triples + lines + planes) / triples
    assert 1.0 < per_triple < 3.0


@pytest.mark.parametrize("mu", [0.0, 3.0])
def test_oracle_line_order_apply_matches_per_triple_order(oracle_mod, mu):
    """A whole adaptive apply with every output node summed in line order gives the same tree and,
    up to FP64 rounding, the same coefficients as the per-triple order, over the same triples
    (including triples whose input is a generated scaling-only block)."""
    O = oracle_mod
    prec = 1e-4
    m = O.MultiResolutionAnalysis(*WORLD, 5, 10)
    f = O.FunctionTree(m)
    O.project(prec, f, O.gauss_params([1.0, -0.3, 0.5], [4.0, 60.0, 15.0],
                                      [(0.1, -0.2, 0.3), (-0.4, 0.2, 0.0), (0.6, 0.5, -0.3)]))
    op = O.PoissonOperator(m, prec) if mu == 0.0 else O.HelmholtzOperator(m, mu, prec)
    a, b = O.FunctionTree(m), O.FunctionTree(m)
    sa = O.apply(prec, a, op, f)
    sb = O.apply_line_ordered(prec, b, op, f)
    assert sa == sb  # triples, triples with generated inputs, passes
    if mu > 0.0:
        assert sa[1] > 0  # this case covers generated inputs
    ea, eb = a.export(), b.export()
    for key in ("depth", "trans", "parent", "child0"):
        assert np.array_equal(ea[key], eb[key]), key
    scale = np.abs(ea["coef"]).max()
    assert np.abs(ea["coef"] - eb["coef"]).max() <= 1e-13 * scale
