"""ctypes front-end of the FP64 CPU oracle (``mw_oracle.cpp``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py``.  The product path never imports it.

The class names mirror the MRCPP objects the reference calls (``MultiResolutionAnalysis``,
``FunctionTree``, ``PoissonOperator``, ``HelmholtzOperator``, ``apply``); see the call sites
``src/qmoperators/two_electron/CoulombPotential.cpp:85`` and
``src/scf_solver/HelmholtzVector.cpp:171-180`` of the reference.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libmworacle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lp = ctypes.POINTER(ctypes.c_longlong)
_vp = ctypes.c_void_p


def build():
    """Compile the oracle library with its Makefile (g++, OpenMP)."""
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.oracle_mra_create.restype = _vp
        L.oracle_mra_create.argtypes = [ctypes.c_int, _ip, _ip, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_mra_destroy.argtypes = [_vp]
        L.oracle_mra_filter.argtypes = [_vp, _dp]
        L.oracle_tree_create.restype = _vp
        L.oracle_tree_create.argtypes = [_vp]
        L.oracle_tree_destroy.argtypes = [_vp]
        L.oracle_project.argtypes = [_vp, ctypes.c_double, ctypes.c_int, _dp]
        L.oracle_tree_nnodes.argtypes = [_vp]
        L.oracle_tree_square_norm.restype = ctypes.c_double
        L.oracle_tree_square_norm.argtypes = [_vp]
        L.oracle_dot.restype = ctypes.c_double
        L.oracle_dot.argtypes = [_vp, _vp]
        L.oracle_evalf.restype = ctypes.c_double
        L.oracle_evalf.argtypes = [_vp, _dp]
        L.oracle_tree_export.argtypes = [_vp, _ip, _lp, _ip, _ip, _dp]
        L.oracle_tree_import.argtypes = [_vp, ctypes.c_int, _ip, _lp, _ip, _ip, _dp]
        L.oracle_operator_create.restype = _vp
        L.oracle_operator_create.argtypes = [_vp, ctypes.c_double, ctypes.c_double]
        L.oracle_operator_destroy.argtypes = [_vp]
        L.oracle_operator_nterms.argtypes = [_vp]
        L.oracle_operator_terms.argtypes = [_vp, _dp, _dp]
        L.oracle_operator_ns.argtypes = [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp]
        L.oracle_scaling_matrix.argtypes = [_vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, _dp]
        L.oracle_apply.argtypes = [ctypes.c_double, _vp, _vp, _vp, _lp]
        L.oracle_apply_ordered.argtypes = [ctypes.c_double, _vp, _vp, _vp, _lp, ctypes.c_int]
        L.oracle_multiply.argtypes = [ctypes.c_double, _vp, ctypes.c_double, _vp, _vp, ctypes.c_int]
        L.oracle_build_grid.argtypes = [_vp, _vp]
        L.oracle_derivative.argtypes = [_vp, _vp, ctypes.c_double, ctypes.c_double, ctypes.c_int]
        L.oracle_add.argtypes = [ctypes.c_double, _vp, ctypes.c_int, _dp, ctypes.POINTER(_vp), ctypes.c_int]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


class MultiResolutionAnalysis:
    """World of ``boxes`` root boxes of edge 2^-min_scale at integer ``corner``
    (reference: ``src/mrenv.cpp:47-72``)."""

    INTERPOLATING = 0
    LEGENDRE = 1

    def __init__(self, min_scale, corner, boxes, order, max_depth, basis=0):
        self.min_scale = int(min_scale)
        self.corner = tuple(int(c) for c in corner)
        self.boxes = tuple(int(b) for b in boxes)
        self.order = int(order)
        self.k = self.order + 1
        self.max_depth = int(max_depth)
        self.basis = int(basis)
        c = (ctypes.c_int * 3)(*self.corner)
        b = (ctypes.c_int * 3)(*self.boxes)
        self._h = lib().oracle_mra_create(self.min_scale, c, b, self.basis, self.order, self.max_depth)

    def filter(self):
        K2 = 2 * self.k
        F = np.zeros((K2, K2))
        lib().oracle_mra_filter(self._h, _d(F))
        return F

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.oracle_mra_destroy(self._h)
            self._h = None


class FunctionTree:
    def __init__(self, mra: MultiResolutionAnalysis):
        self.mra = mra
        self._h = lib().oracle_tree_create(mra._h)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.oracle_tree_destroy(self._h)
            self._h = None

    def nnodes(self):
        return lib().oracle_tree_nnodes(self._h)

    def square_norm(self):
        return lib().oracle_tree_square_norm(self._h)

    def evalf(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        return lib().oracle_evalf(self._h, _d(r))

    def export(self, with_coefs=True):
        n = self.nnodes()
        k = self.mra.k
        depth = np.zeros(n, np.int32)
        trans = np.zeros((n, 3), np.int64)
        parent = np.zeros(n, np.int32)
        child0 = np.zeros(n, np.int32)
        coef = np.zeros((n, 2 * k, 2 * k, 2 * k)) if with_coefs else None
        lib().oracle_tree_export(
            self._h, depth.ctypes.data_as(_ip), trans.ctypes.data_as(_lp), parent.ctypes.data_as(_ip),
            child0.ctypes.data_as(_ip), _d(coef) if with_coefs else None)
        return dict(depth=depth, trans=trans, parent=parent, child0=child0, coef=coef)

    def load(self, depth, trans, parent, child0, coef):
        depth = np.ascontiguousarray(depth, np.int32)
        trans = np.ascontiguousarray(trans, np.int64)
        parent = np.ascontiguousarray(parent, np.int32)
        child0 = np.ascontiguousarray(child0, np.int32)
        coef = np.ascontiguousarray(coef, np.float64)
        lib().oracle_tree_import(self._h, len(depth), depth.ctypes.data_as(_ip), trans.ctypes.data_as(_lp),
                                 parent.ctypes.data_as(_ip), child0.ctypes.data_as(_ip), _d(coef))


def gauss_params(coefs, alphas, centers, powers=None):
    """Parameter block of a Gaussian sum sum_g c_g (r-R_g)^p exp(-alpha_g |r-R_g|^2)."""
    ng = len(coefs)
    p = [float(ng)]
    for g in range(ng):
        pw = (0, 0, 0) if powers is None else powers[g]
        p += [float(coefs[g]), float(alphas[g])] + [float(x) for x in centers[g]] + [float(x) for x in pw]
    return 1, np.array(p)


def hydrogen_params(terms, Z=1.0, origin=(0.0, 0.0, 0.0)):
    """Parameter block of sum_t c_t * phi_{n1 l1 m1}(r) * phi_{n2 l2 m2}(r) (n2 = 0: no second factor).

    Orbitals follow ``src/analyticfunctions/HydrogenFunction.cpp`` of the reference."""
    p = [float(len(terms))]
    for (c, a, b) in terms:
        b = b if b is not None else (0, 0, 0)
        p += [float(c), *map(float, a), *map(float, b), float(Z), *map(float, origin)]
    return 2, np.array(p)


def project(prec, tree: FunctionTree, func):
    ftype, params = func
    params = np.ascontiguousarray(params, np.float64)
    return lib().oracle_project(tree._h, float(prec), int(ftype), _d(params))


def dot(a: FunctionTree, b: FunctionTree):
    return lib().oracle_dot(a._h, b._h)


class ConvolutionOperator:
    def __init__(self, mra, mu, prec):
        self.mra = mra
        self.mu = float(mu)
        self.prec = float(prec)
        self._h = lib().oracle_operator_create(mra._h, self.mu, self.prec)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.oracle_operator_destroy(self._h)
            self._h = None

    def terms(self):
        n = lib().oracle_operator_nterms(self._h)
        a = np.zeros(n)
        b = np.zeros(n)
        lib().oracle_operator_terms(self._h, _d(a), _d(b))
        return a, b

    def ns_matrix(self, depth, term, l):
        K2 = 2 * self.mra.k
        M = np.zeros((K2, K2))
        ok = lib().oracle_operator_ns(self._h, int(depth), int(term), int(l), _d(M))
        return M if ok else None

    def scaling_matrix(self, alpha, n, l):
        k = self.mra.k
        T = np.zeros((k, k))
        lib().oracle_scaling_matrix(self._h, float(alpha), int(n), int(l), _d(T))
        return T


class PoissonOperator(ConvolutionOperator):
    """Kernel 1/|r| (reference: ``src/SCFDriver.cpp:279``)."""

    def __init__(self, mra, prec):
        super().__init__(mra, 0.0, prec)


class HelmholtzOperator(ConvolutionOperator):
    """Kernel exp(-mu|r|)/|r| (reference: ``src/scf_solver/HelmholtzVector.cpp:171``)."""

    def __init__(self, mra, mu, prec):
        super().__init__(mra, mu, prec)


def apply(prec, out: FunctionTree, op: ConvolutionOperator, inp: FunctionTree):
    """Adaptive NS-form apply; returns (triples, triples_with_generated_input, passes)."""
    st = np.zeros(8, np.int64)
    lib().oracle_apply(float(prec), out._h, op._h, inp._h, st.ctypes.data_as(_lp))
    return int(st[0]), int(st[1]), int(st[2])


def apply_line_ordered(prec, out: FunctionTree, op: ConvolutionOperator, inp: FunctionTree):
    """The same apply with every output node's sums taken in the line order of the GPU contraction
    (triples sorted by (term, dz, dy); a line's x products, then a plane's y products, summed before
    the next mode product); returns (triples, triples_with_generated_input, passes)."""
    st = np.zeros(8, np.int64)
    lib().oracle_apply_ordered(float(prec), out._h, op._h, inp._h, st.ctypes.data_as(_lp), 1)
    return int(st[0]), int(st[1]), int(st[2])


def apply_line_stats(prec, out, op, inp):
    """(triples, distinct (node, term, dy, dz) lines, distinct (node, term, dz) planes) of an apply."""
    st = np.zeros(8, np.int64)
    lib().oracle_apply(float(prec), out._h, op._h, inp._h, st.ctypes.data_as(_lp))
    return int(st[0]), int(st[3]), int(st[4])


def multiply(prec, out: FunctionTree, c, a: FunctionTree, b: FunctionTree, max_iter=-1):
    """out = c a b (mrcpp::multiply contract: qmfunction_utils.cpp:209-217, ExchangePotential.cpp:131);
    returns the number of output nodes"""
    return lib().oracle_multiply(float(prec), out._h, float(c), a._h, b._h, int(max_iter))


def build_grid(out: FunctionTree, inp: FunctionTree):
    """extend the grid of `out` by that of `inp` (mrcpp::build_grid, qmfunction_utils.cpp:211-212)"""
    return lib().oracle_build_grid(out._h, inp._h)


def add(prec, out: FunctionTree, coefs, trees, max_iter=-1):
    """out = sum_i coefs[i] trees[i] (mrcpp::add contract, qmfunction_utils.cpp:170-177); returns the
    number of output nodes"""
    n = len(trees)
    c = np.ascontiguousarray(coefs, dtype=np.float64)
    arr = (_vp * n)(*[t._h for t in trees])
    return lib().oracle_add(float(prec), out._h, n, _d(c), arr, int(max_iter))


def derivative(out: FunctionTree, inp: FunctionTree, a, b, direction):
    """out = d/dx_dir inp on the input's grid (ABGV derivative, mrcpp::apply(out, D, inp, dir) contract)"""
    return lib().oracle_derivative(out._h, inp._h, float(a), float(b), int(direction))
