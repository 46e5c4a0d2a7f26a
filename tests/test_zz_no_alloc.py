"""The allocation-free inner product (mw_nalloc_dot) agrees with mw_dot.

mw_nalloc_dot exists for callers that cannot allocate device memory when they need an inner
product (for example under a pre-reserved memory budget, or with the device pool owned by another
framework); it keeps its scratch in a fixed array compiled into the library.  This file runs last (pytest collects files
in name order) and also passes on its own in a fresh process.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WORLD = (-2, (-5, -5, -5), (10, 10, 10))
REL_TOL = 1e-12  # the dot-product tolerance of the other GPU tests


def _tree(G, m, coefs, alphas, centers, prec):
    t = G.FunctionTree(m)
    G.project(prec, t, G.gauss_params(coefs, alphas, centers))
    return t


def test_nalloc_dot_matches_dot_on_consecutive_calls(gpu_mod):
    G = gpu_mod
    m = G.MultiResolutionAnalysis(*WORLD, 7, 12)
    a = _tree(G, m, [1.0, 0.5], [10.0, 3.0], [(0.1, -0.2, 0.3), (-0.5, 0.4, 0.0)], 1e-5)
    b = _tree(G, m, [2.0], [1.5], [(0.2, 0.0, -0.1)], 1e-5)
    c = _tree(G, m, [0.7, -0.3], [40.0, 0.8], [(1.0, 1.0, 0.0), (-1.0, 0.5, 0.5)], 1e-5)

    # first call (also performs the one-time device set-up), then further calls in a row
    first = G.nalloc_dot(a, b)
    second = G.nalloc_dot(c, a)
    third = G.nalloc_dot(a, b)
    for got, (x, y) in ((first, (a, b)), (second, (c, a)), (third, (a, b))):
        ref = G.dot(x, y)
        assert np.isfinite(got)
        assert abs(got - ref) <= REL_TOL * abs(ref), (got, ref)
    # the shared scratch keeps no state between calls
    assert first == third


def test_nalloc_dot_rejects_mismatched_worlds(gpu_mod):
    G = gpu_mod
    m1 = G.MultiResolutionAnalysis(*WORLD, 5, 10)
    m2 = G.MultiResolutionAnalysis(*WORLD, 5, 10)
    a = _tree(G, m1, [1.0], [1.0], [(0.0, 0.0, 0.0)], 1e-3)
    b = _tree(G, m2, [1.0], [1.0], [(0.0, 0.0, 0.0)], 1e-3)
    with pytest.raises(G.MWError):
        G.nalloc_dot(a, b)
