"""Python mirror of the MRCPP operator-apply interface, bound to the C-ABI library ``libmwb200.so``.

Names and argument meaning follow the objects the reference calls on this path:

* ``MultiResolutionAnalysis(min_scale, corner, boxes, order, max_depth, basis)`` --
  ``BoundingBox<3>`` + ``InterpolatingBasis``/``LegendreBasis`` + ``MultiResolutionAnalysis<3>``
  (reference ``src/mrenv.cpp:52,64-72``);
* ``FunctionTree(mra)`` -- ``FunctionTree<3>`` (``src/qmfunctions/QMFunction.cpp:68-77``);
* ``PoissonOperator(mra, prec)`` / ``HelmholtzOperator(mra, mu, prec)``
  (``src/SCFDriver.cpp:279``, ``src/scf_solver/HelmholtzVector.cpp:171``);
* ``apply(prec, out, op, inp)`` (``src/scf_solver/HelmholtzVector.cpp:176``,
  ``src/qmoperators/two_electron/CoulombPotential.cpp:85``);
* ``project(prec, tree, f)`` and ``dot(a, b)``.

Every call runs on the GPU through the C-ABI; there is no CPU path.  A non-zero status from the
library raises :class:`MWError` (the reference aborts through ``MSG_FATAL`` instead).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmwb200.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lp = ctypes.POINTER(ctypes.c_longlong)
_vp = ctypes.c_void_p
_vpp = ctypes.POINTER(ctypes.c_void_p)
_fp = ctypes.POINTER(ctypes.c_float)

BASIS_INTERPOLATING = 0
BASIS_LEGENDRE = 1
FUNC_GAUSSIANS = 1
FUNC_HYDROGEN_PRODUCTS = 2
APPLY_FP64 = 0
APPLY_FP32 = 1
APPLY_TF32X3 = 2  # split-TF32 tensor cores (k <= 10, prec >= 1e-6; otherwise the FP32 engine)
APPLY_BF16X3 = 3  # x step on the tensor cores (BF16 slices: 4 per data row, 3 per operator row), y/z FP32, FP64 sums (k = 7..10)

# every symbol include/mwb200.h declares: (name, restype, argtypes)
SYMBOLS = [
    ("mw_last_error", ctypes.c_char_p, []),
    ("mw_version", ctypes.c_int, [_ip, _ip]),
    ("mw_ctx_create", ctypes.c_int, [ctypes.c_int, _vp, _vpp]),
    ("mw_ctx_destroy", ctypes.c_int, [_vp]),
    ("mw_ctx_synchronize", ctypes.c_int, [_vp]),
    ("mw_ctx_reserve", ctypes.c_int, [_vp, ctypes.c_ulonglong]),
    ("mw_tree_assign", ctypes.c_int, [_vp, _vp]),
    ("mw_ctx_set_chunk_triples", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    ("mw_ctx_get_chunk_triples", ctypes.c_int, [_vp, ctypes.c_int, _ip]),
    ("mw_ctx_profile", ctypes.c_int, [_vp, ctypes.c_int]),
    ("mw_ctx_profile_read", ctypes.c_int, [_vp, _lp, _lp, _dp]),
    ("mw_ctx_profile_ctas", ctypes.c_int, [_vp, _lp]),
    ("mw_mra_create", ctypes.c_int, [_vp, ctypes.c_int, _ip, _ip, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vpp]),
    ("mw_mra_destroy", ctypes.c_int, [_vp]),
    ("mw_mra_filter", ctypes.c_int, [_vp, _dp]),
    ("mw_op_scaling_matrix", ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_int, ctypes.c_longlong, _dp]),
    ("mw_op_ns_matrix", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_longlong, _dp]),
    ("mw_mra_max_depth", ctypes.c_int, [_vp, _ip]),
    ("mw_tree_create", ctypes.c_int, [_vp, _vpp]),
    ("mw_tree_destroy", ctypes.c_int, [_vp]),
    ("mw_tree_nnodes", ctypes.c_int, [_vp, _ip]),
    ("mw_tree_square_norm", ctypes.c_int, [_vp, _dp]),
    ("mw_tree_upload", ctypes.c_int, [_vp, ctypes.c_int, _ip, _lp, _ip, _ip, _dp]),
    ("mw_tree_download", ctypes.c_int, [_vp, _ip, _lp, _ip, _ip, _dp]),
    ("mw_tree_upload_many", ctypes.c_int, [ctypes.c_int, _vpp, _ip, _vpp, _vpp, _vpp, _vpp, _vpp]),
    ("mw_tree_download_many", ctypes.c_int, [ctypes.c_int, _vpp, _vpp, _vpp, _vpp, _vpp, _vpp]),
    ("mw_tree_device_arrays", ctypes.c_int, [_vp, _vpp, _vpp, _vpp]),
    ("mw_tree_rescale", ctypes.c_int, [_vp, ctypes.c_double]),
    ("mw_tree_serialized_size", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_ulonglong)]),
    ("mw_tree_serialize", ctypes.c_int, [_vp, _vp, ctypes.c_ulonglong]),
    ("mw_tree_deserialize", ctypes.c_int, [_vp, _vp, ctypes.c_ulonglong]),
    ("mw_tree_save", ctypes.c_int, [_vp, ctypes.c_char_p]),
    ("mw_tree_load", ctypes.c_int, [_vp, ctypes.c_char_p]),
    ("mw_project", ctypes.c_int, [ctypes.c_double, _vp, ctypes.c_int, ctypes.c_int, _dp]),
    ("mw_dot", ctypes.c_int, [_vp, _vp, _dp]),
    ("mw_nalloc_dot", ctypes.c_int, [_vp, _vp, _dp]),
    ("mw_tree_distance", ctypes.c_int, [_vp, _vp, _dp]),
    ("mw_op_create_poisson", ctypes.c_int, [_vp, ctypes.c_double, _vpp]),
    ("mw_op_create_helmholtz", ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, _vpp]),
    ("mw_op_create_abgv", ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, _vpp]),
    ("mw_apply_derivative", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int]),
    ("mw_op_destroy", ctypes.c_int, [_vp]),
    ("mw_op_nterms", ctypes.c_int, [_vp, _ip]),
    ("mw_op_terms", ctypes.c_int, [_vp, _dp, _dp]),
    ("mw_apply", ctypes.c_int, [ctypes.c_double, _vp, _vp, _vp, ctypes.c_int]),
    ("mw_apply_batched", ctypes.c_int, [ctypes.c_int, ctypes.c_double, _vpp, _vpp, _vpp, ctypes.c_int]),
    ("mw_apply_stats", ctypes.c_int, [_vp, _lp]),
    ("mw_multiply", ctypes.c_int, [ctypes.c_double, _vp, ctypes.c_double, _vp, _vp, ctypes.c_int]),
    ("mw_multiply_batched", ctypes.c_int, [ctypes.c_int, ctypes.c_double, _vpp, _dp, _vpp, _vpp, ctypes.c_int]),
    ("mw_square", ctypes.c_int, [ctypes.c_double, _vp, _vp, ctypes.c_int]),
    ("mw_tree_build_grid", ctypes.c_int, [_vp, _vp]),
    ("mw_add", ctypes.c_int, [ctypes.c_double, _vp, ctypes.c_int, _dp, _vpp, ctypes.c_int]),
    ("mw_tree_copy_grid", ctypes.c_int, [_vp, _vp]),
    ("mw_tree_clear", ctypes.c_int, [_vp]),
    ("mw_mlp_create", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_uint, _vpp]),
    ("mw_mlp_destroy", ctypes.c_int, [_vp]),
    ("mw_mlp_nparams", ctypes.c_int, [_vp, _lp, _ip]),
    ("mw_mlp_get_params", ctypes.c_int, [_vp, _fp]),
    ("mw_mlp_set_params", ctypes.c_int, [_vp, _fp]),
    ("mw_mlp_forward", ctypes.c_int, [_vp, ctypes.c_int, _fp, _fp]),
    ("mw_mlp_gradient", ctypes.c_int, [_vp, ctypes.c_int, _fp, _fp, _fp, _dp, _fp]),
    ("mw_mlp_collect", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("mw_mlp_dataset", ctypes.c_int, [_vp, _ip, _ip]),
    ("mw_mlp_dataset_get", ctypes.c_int, [_vp, _fp, _fp]),
    ("mw_mlp_train", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_uint, _dp]),
    ("mw_apply_learned", ctypes.c_int, [ctypes.c_int, ctypes.c_double, _vpp, _vpp, _vpp, ctypes.c_int, _vp,
                                         ctypes.c_float, _lp]),
]

_lib = None


class MWError(RuntimeError):
    """Error status returned by the C-ABI."""


def load_library(path: str = LIB_PATH):
    """Load ``libmwb200.so`` and bind every declared symbol; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"libmwb200.so not built ({path}); run __graft_entry__.build()")
    L = ctypes.CDLL(path)
    for name, res, args in SYMBOLS:
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _check(status):
    if status != 0:
        msg = _lib.mw_last_error().decode(errors="replace")
        raise MWError(f"mwb200 error {status}: {msg}")


def _d(a):
    return a.ctypes.data_as(_dp)


class Context:
    """CUDA device + stream + memory pool of the library."""

    _default = None

    def __init__(self, device: int = 0, stream: int | None = None):
        L = load_library()
        h = ctypes.c_void_p()
        _check(L.mw_ctx_create(int(device), stream, ctypes.byref(h)))
        self._h = h
        self.device = device

    @classmethod
    def default(cls):
        if cls._default is None:
            cls._default = Context(0)
        return cls._default

    def synchronize(self):
        _check(_lib.mw_ctx_synchronize(self._h))

    def reserve(self, nbytes):
        """Grow the device memory pool to at least nbytes up front (see mw_ctx_reserve)."""
        _check(_lib.mw_ctx_reserve(self._h, int(nbytes)))

    def set_chunk_triples(self, flags, triples):
        """Contraction work per CTA for applies under `flags` (see mw_ctx_set_chunk_triples)."""
        _check(_lib.mw_ctx_set_chunk_triples(self._h, int(flags), int(triples)))

    def chunk_triples(self, flags):
        v = ctypes.c_int()
        _check(_lib.mw_ctx_get_chunk_triples(self._h, int(flags), ctypes.byref(v)))
        return v.value

    def profile(self, enable=True):
        """Reset and (de)activate the kernel counters."""
        _check(_lib.mw_ctx_profile(self._h, int(enable)))

    def profile_ctas(self):
        """contraction CTAs launched since profile()"""
        v = ctypes.c_longlong()
        _check(_lib.mw_ctx_profile_ctas(self._h, ctypes.byref(v)))
        return v.value

    def profile_read(self):
        """(kernels launched, contraction launches, contraction CUDA-event ms) since profile()."""
        a, b, c = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_double()
        _check(_lib.mw_ctx_profile_read(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value


class MultiResolutionAnalysis:
    INTERPOLATING = BASIS_INTERPOLATING
    LEGENDRE = BASIS_LEGENDRE

    def __init__(self, min_scale, corner, boxes, order, max_depth, basis=BASIS_INTERPOLATING, ctx=None):
        L = load_library()
        self.ctx = ctx or Context.default()
        self.min_scale = int(min_scale)
        self.corner = tuple(int(c) for c in corner)
        self.boxes = tuple(int(b) for b in boxes)
        self.order = int(order)
        self.k = self.order + 1
        self.max_depth = int(max_depth)
        self.basis = int(basis)
        h = ctypes.c_void_p()
        _check(L.mw_mra_create(self.ctx._h, self.min_scale, (ctypes.c_int * 3)(*self.corner),
                               (ctypes.c_int * 3)(*self.boxes), self.basis, self.order, self.max_depth,
                               ctypes.byref(h)))
        self._h = h

    def filter(self):
        F = np.zeros((2 * self.k, 2 * self.k))
        _check(_lib.mw_mra_filter(self._h, _d(F)))
        return F

    def depth_limit(self):
        d = ctypes.c_int()
        _check(_lib.mw_mra_max_depth(self._h, ctypes.byref(d)))
        return d.value

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.mw_mra_destroy(self._h)
            self._h = None


class FunctionTree:
    def __init__(self, mra: MultiResolutionAnalysis):
        self.mra = mra
        h = ctypes.c_void_p()
        _check(load_library().mw_tree_create(mra._h, ctypes.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.mw_tree_destroy(self._h)
            self._h = None

    def nnodes(self):
        n = ctypes.c_int()
        _check(_lib.mw_tree_nnodes(self._h, ctypes.byref(n)))
        return n.value

    getNNodes = nnodes

    def square_norm(self):
        v = ctypes.c_double()
        _check(_lib.mw_tree_square_norm(self._h, ctypes.byref(v)))
        return v.value

    getSquareNorm = square_norm

    def rescale(self, c):
        _check(_lib.mw_tree_rescale(self._h, float(c)))

    def export(self, with_coefs=True):
        n = self.nnodes()
        k = self.mra.k
        depth = np.zeros(n, np.int32)
        trans = np.zeros((n, 3), np.int64)
        parent = np.zeros(n, np.int32)
        child0 = np.zeros(n, np.int32)
        coef = np.zeros((n, 2 * k, 2 * k, 2 * k)) if with_coefs else None
        _check(_lib.mw_tree_download(self._h, depth.ctypes.data_as(_ip), trans.ctypes.data_as(_lp),
                                     parent.ctypes.data_as(_ip), child0.ctypes.data_as(_ip),
                                     _d(coef) if with_coefs else None))
        return dict(depth=depth, trans=trans, parent=parent, child0=child0, coef=coef)

    def serialize(self):
        """flat byte image of the tree (numpy uint8): checkpoint / message payload"""
        n = ctypes.c_ulonglong()
        _check(_lib.mw_tree_serialized_size(self._h, ctypes.byref(n)))
        buf = np.empty(n.value, np.uint8)
        _check(_lib.mw_tree_serialize(self._h, buf.ctypes.data_as(ctypes.c_void_p), n.value))
        return buf

    def deserialize(self, buf):
        """replace the tree by a byte image written on the same world and basis"""
        b = np.ascontiguousarray(buf, dtype=np.uint8)
        _check(_lib.mw_tree_deserialize(self._h, b.ctypes.data_as(ctypes.c_void_p), b.size))

    def save_tree(self, path):
        """FunctionTree::saveTree (reference src/qmfunctions/Orbital.cpp:128)"""
        _check(_lib.mw_tree_save(self._h, os.fsencode(path)))

    def load_tree(self, path):
        """FunctionTree::loadTree (reference src/qmfunctions/Orbital.cpp:170)"""
        _check(_lib.mw_tree_load(self._h, os.fsencode(path)))

    def assign(self, src):
        """self = a deep copy of `src`, device to device; `src` may live in another context (stream) of the
        same device, on a world with the same parameters (see mw_tree_assign).  Blocking."""
        _check(_lib.mw_tree_assign(self._h, src._h))

    def export_into(self, bufs):
        """Download into caller-owned arrays (e.g. pinned host memory reused across calls): `bufs` has
        int32 'depth', 'parent', 'child0' (>= n), int64 'trans' (>= n x 3) and float64 'coef'
        (>= n x (2k)^3), all C-contiguous; returns n.  Nothing is allocated."""
        n = self.nnodes()
        k = self.mra.k
        need = {"depth": (np.int32, n), "parent": (np.int32, n), "child0": (np.int32, n), "trans": (np.int64, 3 * n),
                "coef": (np.float64, n * (2 * k) ** 3)}
        for name, (dt, size) in need.items():
            a = bufs[name]
            if a.dtype != dt or not a.flags.c_contiguous or a.size < size:
                raise MWError(f"export_into: buffer '{name}' must be C-contiguous {np.dtype(dt).name} of >= {size}")
        _check(_lib.mw_tree_download(self._h, bufs["depth"].ctypes.data_as(_ip), bufs["trans"].ctypes.data_as(_lp),
                                     bufs["parent"].ctypes.data_as(_ip), bufs["child0"].ctypes.data_as(_ip),
                                     _d(bufs["coef"])))
        return n

    def load(self, depth, trans, parent, child0, coef):
        depth = np.ascontiguousarray(depth, np.int32)
        trans = np.ascontiguousarray(trans, np.int64)
        parent = np.ascontiguousarray(parent, np.int32)
        child0 = np.ascontiguousarray(child0, np.int32)
        coef = np.ascontiguousarray(coef, np.float64)
        _check(_lib.mw_tree_upload(self._h, len(depth), depth.ctypes.data_as(_ip), trans.ctypes.data_as(_lp),
                                   parent.ctypes.data_as(_ip), child0.ctypes.data_as(_ip), _d(coef)))

    def device_arrays(self):
        c, k, n = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        _check(_lib.mw_tree_device_arrays(self._h, ctypes.byref(c), ctypes.byref(k), ctypes.byref(n)))
        return c.value, k.value, n.value


def _ptrs(arrays):
    return (ctypes.c_void_p * max(1, len(arrays)))(*[None if a is None else a.ctypes.data for a in arrays])


def load_many(trees, arrays):
    """Upload a batch of host trees in one call (mw_tree_upload_many): ``arrays[i]`` is a dict with the
    arguments of ``FunctionTree.load`` ('depth', 'trans', 'parent', 'child0', 'coef') for ``trees[i]``.
    Same checks and results as one ``load`` per tree; the copies of all trees are queued back to back."""
    if len(trees) != len(arrays):
        raise MWError("load_many: one array set per tree")
    conv = {"depth": np.int32, "trans": np.int64, "parent": np.int32, "child0": np.int32, "coef": np.float64}
    keep = [{k: np.ascontiguousarray(a[k], dt) for k, dt in conv.items()} for a in arrays]
    n = np.array([len(a["depth"]) for a in keep], np.int32)
    _check(_lib.mw_tree_upload_many(len(trees), (ctypes.c_void_p * max(1, len(trees)))(*[t._h for t in trees]),
                                    n.ctypes.data_as(_ip), *[_ptrs([a[k] for a in keep]) for k in conv]))


def export_many_into(trees, bufs):
    """Download a batch of trees in one call (mw_tree_download_many) into caller-owned arrays: ``bufs[i]``
    is a dict as for ``FunctionTree.export_into``.  Returns the node counts."""
    if len(trees) != len(bufs):
        raise MWError("export_many_into: one buffer set per tree")
    names = {"depth": np.int32, "trans": np.int64, "parent": np.int32, "child0": np.int32, "coef": np.float64}
    counts = []
    for t, b in zip(trees, bufs):
        n = t.nnodes()
        k = t.mra.k
        size = {"depth": n, "trans": 3 * n, "parent": n, "child0": n, "coef": n * (2 * k) ** 3}
        for name, dt in names.items():
            a = b[name]
            if a.dtype != dt or not a.flags.c_contiguous or not a.flags.writeable or a.size < size[name]:
                raise MWError(f"export_many_into: buffer '{name}' must be writable C-contiguous "
                              f"{np.dtype(dt).name} of >= {size[name]}")
        counts.append(n)
    _check(_lib.mw_tree_download_many(len(trees), (ctypes.c_void_p * max(1, len(trees)))(*[t._h for t in trees]),
                                      *[_ptrs([b[k] for b in bufs]) for k in names]))
    return counts


def gauss_params(coefs, alphas, centers, powers=None):
    """Parameter block of sum_g c_g (r-R_g)^p exp(-alpha_g |r-R_g|^2) (``GaussExp<3>`` analogue)."""
    ng = len(coefs)
    p = [float(ng)]
    for g in range(ng):
        pw = (0, 0, 0) if powers is None else powers[g]
        p += [float(coefs[g]), float(alphas[g])] + [float(x) for x in centers[g]] + [float(x) for x in pw]
    return FUNC_GAUSSIANS, np.array(p)


def hydrogen_params(terms, Z=1.0, origin=(0.0, 0.0, 0.0)):
    """sum_t c_t phi_a(r) phi_b(r) of hydrogen orbitals (reference ``HydrogenFunction``)."""
    p = [float(len(terms))]
    for (c, a, b) in terms:
        b = b if b is not None else (0, 0, 0)
        p += [float(c), *map(float, a), *map(float, b), float(Z), *map(float, origin)]
    return FUNC_HYDROGEN_PRODUCTS, np.array(p)


def project(prec, tree: FunctionTree, func):
    ftype, params = func
    params = np.ascontiguousarray(params, np.float64)
    _check(_lib.mw_project(float(prec), tree._h, int(ftype), len(params), _d(params)))
    return tree.nnodes()


def dot(a: FunctionTree, b: FunctionTree):
    v = ctypes.c_double()
    _check(_lib.mw_dot(a._h, b._h, ctypes.byref(v)))
    return v.value


def distance(a: FunctionTree, b: FunctionTree):
    """||a - b|| from the coefficient differences (no cancellation)"""
    v = ctypes.c_double()
    _check(_lib.mw_tree_distance(a._h, b._h, ctypes.byref(v)))
    return v.value


def nalloc_dot(a: FunctionTree, b: FunctionTree):
    """<a|b> without any device allocation (for callers that cannot allocate, e.g. while recording a
    CUDA graph); at most 2^20 nodes in `a`; concurrent calls on one GPU must be serialised."""
    v = ctypes.c_double()
    _check(_lib.mw_nalloc_dot(a._h, b._h, ctypes.byref(v)))
    return v.value


class ConvolutionOperator:
    def __init__(self, mra, mu, prec):
        self.mra = mra
        self.mu = float(mu)
        self.prec = float(prec)
        h = ctypes.c_void_p()
        L = load_library()
        if self.mu == 0.0:
            _check(L.mw_op_create_poisson(mra._h, self.prec, ctypes.byref(h)))
        else:
            _check(L.mw_op_create_helmholtz(mra._h, self.mu, self.prec, ctypes.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.mw_op_destroy(self._h)
            self._h = None

    def terms(self):
        n = ctypes.c_int()
        _check(_lib.mw_op_nterms(self._h, ctypes.byref(n)))
        a = np.zeros(n.value)
        b = np.zeros(n.value)
        _check(_lib.mw_op_terms(self._h, _d(a), _d(b)))
        return a, b

    def scaling_matrix(self, alpha, n, l):
        """T^n(l) of exp(-alpha x^2), k x k (see mw_op_scaling_matrix)"""
        k = self.mra.k
        T = np.zeros((k, k))
        _check(_lib.mw_op_scaling_matrix(self._h, float(alpha), int(n), int(l), _d(T)))
        return T

    def ns_matrix(self, term, n, l):
        """non-standard-form matrix of a term at scale n, offset l, 2k x 2k (see mw_op_ns_matrix)"""
        k = self.mra.k
        NS = np.zeros((2 * k, 2 * k))
        _check(_lib.mw_op_ns_matrix(self._h, int(term), int(n), int(l), _d(NS)))
        return NS


class PoissonOperator(ConvolutionOperator):
    """Kernel 1/|r|."""

    def __init__(self, mra, prec):
        super().__init__(mra, 0.0, prec)


class HelmholtzOperator(ConvolutionOperator):
    """Kernel exp(-mu|r|)/|r|."""

    def __init__(self, mra, mu, prec):
        if not mu > 0.0:
            raise MWError("mu must be positive")
        super().__init__(mra, mu, prec)


class ABGVOperator:
    """First derivative with flux parameters a, b (mrcpp::ABGVOperator<3>(MRA, a, b), reference
    src/SCFDriver.cpp:282-283)."""

    def __init__(self, mra, a, b):
        self.mra = mra
        h = ctypes.c_void_p()
        _check(load_library().mw_op_create_abgv(mra._h, float(a), float(b), ctypes.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.mw_op_destroy(self._h)
            self._h = None


def apply_derivative(out: FunctionTree, op: ABGVOperator, inp: FunctionTree, direction, flags=APPLY_FP64):
    """out = d/dx_dir inp on the input's grid: mrcpp::apply(out, D, inp, dir) (reference
    src/qmoperators/one_electron/NablaOperator.cpp:35)."""
    _check(_lib.mw_apply_derivative(out._h, op._h, inp._h, int(direction), int(flags)))


def apply_batched(prec, outs, ops, inps, flags=APPLY_FP64):
    """outs[i] = ops[i] * inps[i] for the whole batch in lock-step passes; returns the batch's
    contracted triple count."""
    n = len(outs)
    if not (len(ops) == n and len(inps) == n):
        raise MWError("batch lists must have equal length")
    arr = lambda objs: (ctypes.c_void_p * n)(*[o._h.value for o in objs])
    _check(_lib.mw_apply_batched(n, float(prec), arr(outs), arr(ops), arr(inps), int(flags)))
    st = np.zeros(4, np.int64)
    _check(_lib.mw_apply_stats(outs[0]._h, st.ctypes.data_as(_lp)))
    return int(st[1])


def apply_stats(out: FunctionTree):
    """(triples of this tree or -1 after a batch, triples of the batch, refinement passes, nodes)."""
    st = np.zeros(8, np.int64)
    _check(_lib.mw_apply_stats(out._h, st.ctypes.data_as(_lp)))
    return tuple(int(x) for x in st[:4])


def apply(prec, out: FunctionTree, op: ConvolutionOperator, inp: FunctionTree, flags=APPLY_FP64):
    """out = op * inp (adaptive); returns (triples, triples_gen, passes, out_nodes)."""
    _check(_lib.mw_apply(float(prec), out._h, op._h, inp._h, int(flags)))
    st = np.zeros(4, np.int64)
    _check(_lib.mw_apply_stats(out._h, st.ctypes.data_as(_lp)))
    return tuple(int(x) for x in st)


def multiply(prec, out: FunctionTree, c, a: FunctionTree, b: FunctionTree, max_iter=-1):
    """out = c a b: mrcpp::multiply(prec, out, c, a, b, maxIter) (reference
    src/qmfunctions/qmfunction_utils.cpp:209-217).  `out` keeps its grid (roots when empty) and is
    refined while leaves fail the wavelet test, at most max_iter passes (-1: until converged)."""
    _check(_lib.mw_multiply(float(prec), out._h, float(c), a._h, b._h, int(max_iter)))


def multiply_batched(prec, outs, coefs, a_trees, b_trees, max_iter=-1):
    """outs[i] = coefs[i] a_trees[i] b_trees[i], refinement passes in lock-step over the batch"""
    n = len(outs)
    if not (len(a_trees) == len(b_trees) == n):
        raise MWError("batch lists must have equal length")
    o = (ctypes.c_void_p * n)(*[t._h.value for t in outs])
    a = (ctypes.c_void_p * n)(*[t._h.value for t in a_trees])
    b = (ctypes.c_void_p * n)(*[t._h.value for t in b_trees])
    c = None if coefs is None else np.ascontiguousarray(coefs, dtype=np.float64)
    _check(_lib.mw_multiply_batched(n, float(prec), o, None if c is None else _d(c), a, b, int(max_iter)))


def square(prec, out: FunctionTree, a: FunctionTree, max_iter=-1):
    """out = a^2: mrcpp::square (reference src/qmfunctions/density_utils.cpp:74)"""
    _check(_lib.mw_square(float(prec), out._h, a._h, int(max_iter)))


def add(prec, out: FunctionTree, coefs, trees, max_iter=-1):
    """out = sum_i coefs[i] trees[i]: mrcpp::add(prec, out, vec, maxIter) (reference
    src/qmfunctions/qmfunction_utils.cpp:170-177); union-grid form: build_grid(out, t) for every tree,
    then prec < 0 or max_iter = 0"""
    n = len(trees)
    if n != len(coefs):
        raise MWError("coefficient and tree lists must have equal length")
    c = np.ascontiguousarray(coefs, dtype=np.float64)
    arr = (ctypes.c_void_p * n)(*[t._h.value for t in trees])
    _check(_lib.mw_add(float(prec), out._h, n, _d(c), arr, int(max_iter)))


def build_grid(out: FunctionTree, inp: FunctionTree):
    """extend the grid of `out` by that of `inp`: mrcpp::build_grid (qmfunction_utils.cpp:211-212)"""
    _check(_lib.mw_tree_build_grid(out._h, inp._h))


def copy_grid(out: FunctionTree, inp: FunctionTree):
    """out gets the grid of inp (blocks zero): mrcpp::copy_grid (density_utils.cpp:73)"""
    _check(_lib.mw_tree_copy_grid(out._h, inp._h))


def clear(tree: FunctionTree):
    """empty the tree"""
    _check(_lib.mw_tree_clear(tree._h))


class ProposalNet:
    """Learned output-tree proposal: an FP32 MLP (hidden_layers x width) on the device, trained by the
    library's own forward/backward/Adam kernels on labels from plain applies."""

    def __init__(self, ctx=None, hidden_layers=3, width=128, seed=0):
        L = load_library()
        self.ctx = ctx or Context.default()
        h = ctypes.c_void_p()
        _check(L.mw_mlp_create(self.ctx._h, int(hidden_layers), int(width), int(seed), ctypes.byref(h)))
        self._h = h
        n, nf = ctypes.c_longlong(), ctypes.c_int()
        _check(L.mw_mlp_nparams(h, ctypes.byref(n), ctypes.byref(nf)))
        self.nparams, self.nfeatures = n.value, nf.value
        self.dims = [self.nfeatures] + [int(width)] * int(hidden_layers) + [1]

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.mw_mlp_destroy(self._h)
            self._h = None

    def params(self):
        p = np.zeros(self.nparams, np.float32)
        _check(_lib.mw_mlp_get_params(self._h, p.ctypes.data_as(_fp)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        _check(_lib.mw_mlp_set_params(self._h, p.ctypes.data_as(_fp)))

    def layers(self, p=None):
        """[(W, b)] views of a parameter vector (W: out x in)."""
        p = self.params() if p is None else p
        out, off = [], 0
        for i in range(len(self.dims) - 1):
            nin, nout = self.dims[i], self.dims[i + 1]
            W = p[off:off + nin * nout].reshape(nout, nin)
            off += nin * nout
            b = p[off:off + nout]
            off += nout
            out.append((W, b))
        return out

    def forward(self, x):
        x = np.ascontiguousarray(x, np.float32)
        z = np.zeros(len(x), np.float32)
        _check(_lib.mw_mlp_forward(self._h, len(x), x.ctypes.data_as(_fp), z.ctypes.data_as(_fp)))
        return z

    def gradient(self, x, y, w):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        w = np.ascontiguousarray(w, np.float32)
        g = np.zeros(self.nparams, np.float32)
        loss = ctypes.c_double()
        _check(_lib.mw_mlp_gradient(self._h, len(x), x.ctypes.data_as(_fp), y.ctypes.data_as(_fp),
                                    w.ctypes.data_as(_fp), ctypes.byref(loss), g.ctypes.data_as(_fp)))
        return loss.value, g

    def collect(self, out, op, inp):
        """Add the split labels of a plain apply (out = op * inp) to the training set."""
        _check(_lib.mw_mlp_collect(self._h, out._h, op._h, inp._h))

    def dataset(self, with_data=False):
        n, npos = ctypes.c_int(), ctypes.c_int()
        _check(_lib.mw_mlp_dataset(self._h, ctypes.byref(n), ctypes.byref(npos)))
        if not with_data:
            return n.value, npos.value
        x = np.zeros((n.value, self.nfeatures), np.float32)
        y = np.zeros(n.value, np.float32)
        _check(_lib.mw_mlp_dataset_get(self._h, x.ctypes.data_as(_fp), y.ctypes.data_as(_fp)))
        return x, y

    def train(self, epochs=20, batch=4096, lr=1e-3, seed=0):
        loss = ctypes.c_double()
        _check(_lib.mw_mlp_train(self._h, int(epochs), int(batch), float(lr), int(seed), ctypes.byref(loss)))
        return loss.value


def apply_learned(prec, outs, ops, inps, net: ProposalNet, tau=0.5, flags=APPLY_FP64):
    """Learned apply of a batch; same result as apply_batched.  Returns dict of statistics."""
    n = len(outs)
    arr = lambda objs: (ctypes.c_void_p * n)(*[o._h.value for o in objs])
    st = np.zeros(8, np.int64)
    _check(_lib.mw_apply_learned(n, float(prec), arr(outs), arr(ops), arr(inps), int(flags), net._h, float(tau),
                                 st.ctypes.data_as(_lp)))
    keys = ["triples", "passes", "proposed", "pruned", "missed", "out_nodes"]
    return {k: int(v) for k, v in zip(keys, st[:6])}
