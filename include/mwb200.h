/* mwb200.h -- C-ABI of the B200-native multiwavelet (MW) operator apply.
 *
 * Plain pointers and sizes only; every entry point returns an int status (0 = ok, < 0 = error) and
 * never throws.  The text of the last error on the calling thread is returned by mw_last_error().
 * The C++ front-end in mrcpp_b200.h maps a non-zero status to the reference's abort convention
 * (MSG_FATAL), and the Python mirror (mrchem_b200/mrcpp.py) maps it to an exception.
 *
 * Each entry point names the reference interface it replaces.  The reference (MRChem) calls these
 * MRCPP functions; MRCPP itself is an un-vendored submodule (.gitmodules:4-6), so the citations are
 * the reference's call sites, which fix the contract.
 *
 * Data layout shared by every tree buffer crossing this boundary:
 *   node i: depth[i] (0 = root scale n0 = min_scale), translation trans[3*i+d] >= 0 relative to the
 *   world corner at that depth, parent[i] (-1 for roots), child0[i] (index of the first of 8
 *   consecutive children, child c = cx + 2 cy + 4 cz; -1 for leaves), and coef[i*(2k)^3 ...]: the
 *   node block as a (2k)^3 tensor, x fastest, per-dimension index a = c*k + j with c = 0 scaling /
 *   1 wavelet (compressed form).  Parents precede children.
 */
#ifndef MWB200_H
#define MWB200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mw_ctx_s* mw_ctx;   /* device + stream + memory pool */
typedef struct mw_mra_s* mw_mra;   /* world, basis, filters (host and device copies) */
typedef struct mw_tree_s* mw_tree; /* one function: device SoA node arrays + hash index */
typedef struct mw_op_s* mw_op;     /* separated-Gaussian convolution operator, device tables */
typedef struct mw_mlp_s* mw_mlp;   /* learned output-tree proposal network (FP32 MLP on the device) */

enum { MW_OK = 0, MW_ERR_ARG = -1, MW_ERR_CUDA = -2, MW_ERR_STATE = -3, MW_ERR_CAPACITY = -4 };
enum { MW_BASIS_INTERPOLATING = 0, MW_BASIS_LEGENDRE = 1 };
enum { MW_FUNC_GAUSSIANS = 1, MW_FUNC_HYDROGEN_PRODUCTS = 2 };
/* apply flags: FP64 products (the plain apply), or FP32 products with every term's contribution
 * accumulated in FP64 (mixed precision), or split-TF32 products on the tensor cores (data in two TF32
 * pieces, operators in three; FP32 sums inside a term, compensated summation over terms; relative
 * error 2e-7 .. 1e-6, so it serves orders k <= 10 at prec >= 1e-6 (where its error is at most about
 * prec), and other requests take the FP32 path), or BF16x3: the x mode product of every
 * (output, input, term) triple on the tensor cores with data rows as four and operator rows as three
 * BF16 slices of a per-row fixed-point form (exact FP32 sums of each slice pair inside a triple;
 * FP32-level error), the y and z mode
 * products as FP32 products on the CUDA cores and every term's contribution accumulated in FP64 (orders
 * k = 7 .. 10; other orders take the FP32 path); norms, screening and refinement are FP64 in all four */
enum { MW_APPLY_FP64 = 0, MW_APPLY_FP32 = 1, MW_APPLY_TF32X3 = 2, MW_APPLY_BF16X3 = 3 };

const char* mw_last_error(void);
int mw_version(int* major, int* minor);

/* Device context on CUDA device `device`; work is issued on `stream` (NULL = a private stream).  A
 * context (and every handle on it) is used by one host thread at a time: its calls share the stream,
 * the memory pool's stream order and a pinned staging buffer for small uploads.  Threads that work
 * concurrently use one context each. */
int mw_ctx_create(int device, void* stream, mw_ctx* out);
int mw_ctx_destroy(mw_ctx ctx);
int mw_ctx_synchronize(mw_ctx ctx);
/* Grow the context's device memory pool to at least `bytes` once, up front.  Every allocation of the
 * library is stream-ordered from the device's default pool, which keeps freed memory (release
 * threshold: unlimited); a pool that must still grow maps new memory inside the first calls that
 * need it, which makes their time vary.  Reserving the working set once removes that. */
int mw_ctx_reserve(mw_ctx ctx, unsigned long long bytes);
/* Contraction work per CTA of the context's applies under `flags` (one of MW_APPLY_*): each output
 * node's (input node, term) pairs are cut into chunks of at most `triples` (1 .. 4096; default 48),
 * one CTA each; more triples per CTA mean fewer partial blocks to reduce, fewer mean better load
 * balance.  Results agree to FP64 rounding for any value (the partial sums are regrouped).  No
 * reference counterpart (MRCPP schedules with OpenMP); set by mrchem_b200.autotune or the caller. */
int mw_ctx_set_chunk_triples(mw_ctx ctx, int flags, int triples);
int mw_ctx_get_chunk_triples(mw_ctx ctx, int flags, int* triples);
/* Benchmark counters (no reference counterpart: the reference times with mrcpp::Timer around whole
 * calls, src/scf_solver/HelmholtzVector.cpp:68-82).  enable != 0 resets and starts them: number of
 * kernels this library launched, and number and CUDA-event time (ms) of contraction-kernel launches. */
int mw_ctx_profile(mw_ctx ctx, int enable);
int mw_ctx_profile_read(mw_ctx ctx, long long* launches, long long* apply_launches, double* apply_ms);
/* CTAs (chunks of <= chunk_triples triples of one output node) of the contraction launches counted since
 * mw_ctx_profile(ctx, 1): the unit the contraction's DRAM traffic scales with */
int mw_ctx_profile_ctas(mw_ctx ctx, long long* ctas);

/* World and basis.  Replaces BoundingBox<3>(min_scale, corner, boxes) +
 * InterpolatingBasis(order) / LegendreBasis(order) + MultiResolutionAnalysis<3>(world, basis,
 * max_depth): reference src/mrenv.cpp:52,64-72 and tests/unit_tests.cpp:36-43. */
int mw_mra_create(mw_ctx ctx, int min_scale, const int* corner, const int* boxes, int basis_type,
                  int order, int max_depth, mw_mra* out);
int mw_mra_destroy(mw_mra mra);
/* (2k)x(2k) two-scale filter [[H0 H1];[G0 G1]], row-major */
int mw_mra_filter(mw_mra mra, double* F);
/* effective depth limit (max_depth clamped to the 19-bit translation key) */
int mw_mra_max_depth(mw_mra mra, int* depth);

/* Function trees.  Replaces FunctionTree<3>(const MRA&): reference src/qmfunctions/QMFunction.cpp:68-77. */
int mw_tree_create(mw_mra mra, mw_tree* out);
int mw_tree_destroy(mw_tree tree);
/* getNNodes / getSquareNorm: reference src/scf_solver/HelmholtzVector.cpp:84-89 */
int mw_tree_nnodes(mw_tree tree, int* n);
int mw_tree_square_norm(mw_tree tree, double* out);
/* copy a host tree (layout above) to the device; builds the hash index and norms */
int mw_tree_upload(mw_tree tree, int n, const int* depth, const long long* trans, const int* parent,
                   const int* child0, const double* coef);
/* copy the device tree to host buffers sized with mw_tree_nnodes (any pointer may be NULL) */
int mw_tree_download(mw_tree tree, int* depth, long long* trans, int* parent, int* child0, double* coef);
/* Batched transfers of ntrees distinct trees (arrays of per-tree pointers; n[i] nodes for tree i): the
 * same checks, node order and results as mw_tree_upload / mw_tree_download for every tree, with the
 * copies of all trees queued back to back and one synchronisation per call, so that the copy engine
 * streams a whole batch from or to pinned host buffers without idling between trees.  The upload checks
 * every tree before it queues any copy.  The download's trans[i] (3 n_i words) also receives the keys
 * before they are expanded in place; entries of depth/trans/parent/child0/coef may be NULL as in
 * mw_tree_download.  No reference counterpart (MRCPP keeps its trees in host memory). */
int mw_tree_upload_many(int ntrees, mw_tree* trees, const int* n, const int* const* depth,
                        const long long* const* trans, const int* const* parent, const int* const* child0,
                        const double* const* coef);
int mw_tree_download_many(int ntrees, mw_tree* trees, int* const* depth, long long* const* trans,
                          int* const* parent, int* const* child0, double* const* coef);
/* dst = a deep copy of src (structure, coefficients, norms), device to device.  The two trees may
 * belong to different contexts (streams) of the same device, on worlds with the same parameters: a
 * thread that streams trees to or from the host on its own context hands them to the context that
 * computes without a host round trip.  Blocking: returns when dst is complete and src may change.
 * No reference counterpart (MRCPP's FunctionTree copy stays in host memory). */
int mw_tree_assign(mw_tree dst, mw_tree src);
/* device pointers of the node arrays (coef: n*(2k)^3 doubles, key: n uint64, norm2: n doubles) */
int mw_tree_device_arrays(mw_tree tree, void** coef, void** key, void** norm2);
/* Flat byte image of a tree: a 64-byte header (magic "MWB2TREE", format version, k, basis type, root
 * scale, corner[3], boxes[3], node count) then int64 trans[3n], float64 coef[n (2k)^3], int32 depth[n],
 * parent[n], child0[n] in the layout above; it is the checkpoint file of mw_tree_save and the payload
 * a caller sends between processes.  Replaces FunctionTree::saveTree / loadTree (reference
 * src/qmfunctions/Orbital.cpp:118-190) and the payload of mrcpp::send_tree / recv_tree
 * (src/parallel.cpp:208-232).  Deserializing checks that the image was written on the same world and
 * basis. */
int mw_tree_serialized_size(mw_tree tree, unsigned long long* bytes);
int mw_tree_serialize(mw_tree tree, void* buf, unsigned long long cap);
int mw_tree_deserialize(mw_tree tree, const void* buf, unsigned long long len);
int mw_tree_save(mw_tree tree, const char* path);
int mw_tree_load(mw_tree tree, const char* path);
/* rescale(c): reference src/scf_solver/HelmholtzVector.cpp:81 (out[i].rescale(-1/2pi)) */
int mw_tree_rescale(mw_tree tree, double c);

/* Adaptive projection of an analytic function on the device.  Replaces mrcpp::project(prec, tree, f):
 * reference src/qmfunctions/qmfunction_utils.cpp:88-114, src/initial_guess/gto.cpp:159.
 *   MW_FUNC_GAUSSIANS: params = [ng, then per Gaussian: c, alpha, X, Y, Z, px, py, pz]
 *     f(r) = sum c (x-X)^px (y-Y)^py (z-Z)^pz exp(-alpha |r-R|^2)
 *   MW_FUNC_HYDROGEN_PRODUCTS: params = [nt, then per term: c, n1, l1, m1, n2, l2, m2, Z, ox, oy, oz]
 *     f(r) = sum c phi_{n1 l1 m1}(r) phi_{n2 l2 m2}(r) (n2 = 0: no second factor), orbitals as in
 *     reference src/analyticfunctions/HydrogenFunction.cpp:28-160. */
int mw_project(double prec, mw_tree tree, int func_type, int nparams, const double* params);

/* Inner product <a|b> of two compressed trees (reference: orbital::dot via mrcpp::dot,
 * tests/qmoperators/coulomb_operator.cpp:90). */
int mw_dot(mw_tree a, mw_tree b, double* out);

/* ||a - b|| (L2 norm of the difference of two compressed trees on one world, any grids; a node that
 * one tree lacks counts with zero wavelets there).  Computed from the coefficient differences, so it
 * resolves differences far below the cancellation limit of ||a||^2 + ||b||^2 - 2<a|b>.  Used to
 * report the error of the mixed-precision apply against the FP64 one. */
int mw_tree_distance(mw_tree a, mw_tree b, double* out);

/* Allocation-free inner product <a|b>.  No counterpart in the reference: it serves callers that
 * cannot allocate device memory when they need the result -- code under a fixed, pre-reserved memory
 * budget, a host whose device memory pool belongs to another framework, or a thread that must leave
 * the allocator alone while other work on its device is being recorded.  The call itself ends with a
 * blocking read of the result, so it is not made inside a stream capture.  Same result as mw_dot (which allocates two
 * small scratch buffers per call), computed with a fixed scratch array compiled into the library:
 * 8 MiB per GPU that loads the library, held until process exit.
 *   - `a` may have at most 1048576 (2^20) nodes; larger trees return MW_ERR_CAPACITY.
 *   - The first call on a device looks up the array's device address; make that first call before
 *     any stream capture on that device.
 *   - Every call shares the one array: calls that overlap on the GPU (other streams, other threads)
 *     race and must be serialised by the caller.
 *   - `out` is a host pointer; the call returns after the result is written. */
int mw_nalloc_dot(mw_tree a, mw_tree b, double* out);

/* Convolution operators.  Replace mrcpp::PoissonOperator(MRA, prec) (reference src/SCFDriver.cpp:279,
 * tests/qmoperators/coulomb_operator.cpp:84) and mrcpp::HelmholtzOperator(MRA, mu, prec)
 * (reference src/scf_solver/HelmholtzVector.cpp:171).  Kernels 1/|r| and exp(-mu|r|)/|r|. */
int mw_op_create_poisson(mw_mra mra, double prec, mw_op* out);
int mw_op_create_helmholtz(mw_mra mra, double mu, double prec, mw_op* out);
/* First-derivative operator with numerical flux parameters a, b in [0, 1] (Alpert, Beylkin, Gines &
 * Vozovoi 2002; a = b = 0: the cell-local derivative, a = b = 1/2: central flux).  Replaces
 * mrcpp::ABGVOperator<3>(MRA, a, b): reference src/SCFDriver.cpp:282-283, src/mrdft/XCFunctional.cpp:67. */
int mw_op_create_abgv(mw_mra mra, double a, double b, mw_op* out);
/* out = d/dx_dir inp (dir 0, 1, 2 = x, y, z) on the input's grid (no refinement).  Replaces
 * mrcpp::apply(out, D, inp, dir): reference src/qmoperators/one_electron/NablaOperator.cpp:35,40,
 * MomentumOperator.cpp:35,41.  `out` is overwritten and left compressed with valid norms. */
int mw_apply_derivative(mw_tree out, mw_op op, mw_tree inp, int dir, int flags);
int mw_op_destroy(mw_op op);
int mw_op_nterms(mw_op op, int* n);
int mw_op_terms(mw_op op, double* alpha, double* beta);
/* The operator's 1-D matrices as the contraction uses them (for verification against independent
 * quadrature; no reference counterpart, MRCPP keeps them internal to its OperatorCalculator):
 * T^n(l) (k x k, row-major) of exp(-alpha x^2) between scaling functions at scale n, translation
 * offset l -- entry (i, j) = 2^-n int_0^1 int_0^1 phi_i(u) phi_j(v) exp(-alpha 4^-n (u - v + l)^2);
 * and the non-standard-form matrix (2k x 2k, rows = output scaling|wavelet, columns = input) of term
 * `term` at scale n, offset l: F [[T(2l) T(2l-1)]; [T(2l+1) T(2l)]]_{n+1} F^T with the world's two-scale
 * filter F (mw_mra_filter). */
int mw_op_scaling_matrix(mw_op op, double alpha, int n, long long l, double* T);
int mw_op_ns_matrix(mw_op op, int term, int n, long long l, double* NS);

/* out = op * inp, adaptive.  Replaces mrcpp::apply(prec, out, op, inp): reference
 * src/scf_solver/HelmholtzVector.cpp:176,180, src/qmoperators/two_electron/CoulombPotential.cpp:85,
 * src/qmoperators/two_electron/ExchangePotential.cpp:137,259,318.  `out` is overwritten and left
 * compressed with valid norms. */
int mw_apply(double prec, mw_tree out, mw_op op, mw_tree inp, int flags);
/* Batched apply: out[i] = ops[i] * inp[i] for i < n (n <= 128), all on one world; the refinement
 * passes of the whole batch run together (one launch per stage and depth).  Same result per tree as
 * n separate mw_apply calls.  Replaces the per-orbital loop of reference
 * src/scf_solver/HelmholtzVector.cpp:129-135,168-184 (one HelmholtzOperator and one apply per orbital). */
int mw_apply_batched(int n, double prec, mw_tree* out, mw_op* ops, mw_tree* inp, int flags);
/* statistics of the last apply into `out`: [0] contracted (out node, in node, term) triples of this
 * tree (-1 after a batched apply of more than one tree), [1] triples of the whole batch,
 * [2] refinement passes, [3] output nodes */
int mw_apply_stats(mw_tree out, long long* stats);

/* Pointwise product out = c a b.  Replaces mrcpp::multiply(prec, out, c, a, b[, maxIter]):
 * reference src/qmfunctions/qmfunction_utils.cpp:209-217, src/qmoperators/two_electron/ExchangePotential.cpp:
 * 131,253,312.  `out` keeps its current grid (an empty tree starts from the root boxes); every leaf is
 * computed, then leaves whose wavelet norm exceeds prec ||out|| 2^{-depth/2} are split and their
 * children computed, at most max_iter times (max_iter < 0: until no node splits; prec <= 0 or
 * max_iter = 0: the grid is kept, as in the reference's union-grid form).  `out` is left compressed
 * with valid norms.  Orders up to 10 (k <= 11). */
int mw_multiply(double prec, mw_tree out, double c, mw_tree a, mw_tree b, int max_iter);
/* out[i] = c[i] a[i] b[i] for i < n with the refinement passes of the batch in lock-step (c may be NULL:
 * all 1).  Same result per product as n calls of mw_multiply. */
int mw_multiply_batched(int n, double prec, mw_tree* out, const double* c, mw_tree* a, mw_tree* b, int max_iter);
/* out = a^2: mrcpp::square(prec, out, a), reference src/qmfunctions/density_utils.cpp:74 */
int mw_square(double prec, mw_tree out, mw_tree a, int max_iter);
/* Linear combination out = sum_i c[i] f[i] of n <= 256 trees on one world.  Replaces
 * mrcpp::add(prec, out, vec[, maxIter]) with vec = {(c_i, f_i)}: reference
 * src/qmfunctions/qmfunction_utils.cpp:170-177 (qmfunction::linear_combination), density_utils.cpp:87,
 * src/mrdft/XCFunctional.cpp:713, src/scf_solver/KAIN.cpp:180,192.  Grid and refinement as
 * mw_multiply: the union-grid form is mw_tree_build_grid for every f_i, then prec < 0 (or
 * max_iter = 0).  `out` is left compressed with valid norms. */
int mw_add(double prec, mw_tree out, int n, const double* c, mw_tree* f, int max_iter);
/* Grids.  mw_tree_build_grid extends the grid of `out` by that of `inp` (new nodes have zero blocks;
 * mrcpp::build_grid, reference qmfunction_utils.cpp:211-212); mw_tree_copy_grid = clear + build_grid
 * (mrcpp::copy_grid, density_utils.cpp:73); mw_tree_clear empties a tree. */
int mw_tree_build_grid(mw_tree out, mw_tree inp);
int mw_tree_copy_grid(mw_tree out, mw_tree inp);
int mw_tree_clear(mw_tree tree);

/* Learned output-tree proposal.  No counterpart in the reference: MRCPP refines the output tree
 * pass by pass (the plain path above).  A small FP32 MLP predicts which output nodes the wavelet-norm
 * check will split, from 64 features per node (level, position, block and wavelet norms of the 27
 * input neighbours relative to the split threshold, operator and precision scales).  It is trained
 * on the device (forward, backward and Adam kernels of this library) from plain applies. */
int mw_mlp_create(mw_ctx ctx, int hidden_layers, int width, unsigned seed, mw_mlp* out);
int mw_mlp_destroy(mw_mlp mlp);
int mw_mlp_nparams(mw_mlp mlp, long long* n, int* nfeatures);
/* parameters, layer by layer: W (out x in, row-major) then b; host buffers of mw_mlp_nparams floats */
int mw_mlp_get_params(mw_mlp mlp, float* p);
int mw_mlp_set_params(mw_mlp mlp, const float* p);
/* logits of n feature rows (host, n x nfeatures) */
int mw_mlp_forward(mw_mlp mlp, int n, const float* x, float* logits);
/* class-weighted binary cross-entropy of n rows and its gradient w.r.t. all parameters (host) */
int mw_mlp_gradient(mw_mlp mlp, int n, const float* x, const float* y, const float* w, double* loss, float* grad);
/* append the features and split labels of the non-root nodes of `out`, the result of a plain apply of
 * `op` to `inp`, to the network's training set (kept on the device) */
int mw_mlp_collect(mw_mlp mlp, mw_tree out, mw_op op, mw_tree inp);
int mw_mlp_dataset(mw_mlp mlp, int* n, int* npositive);
int mw_mlp_dataset_get(mw_mlp mlp, float* x, float* y);
/* Adam on the training set (class-balanced weights); returns the last epoch's mean loss */
int mw_mlp_train(mw_mlp mlp, int epochs, int batch, float lr, unsigned seed, double* loss);
/* Learned apply: exact root pass, proposal of the deeper tree (nodes with sigmoid(logit) > tau
 * split), one pass over all proposed nodes, then the plain criterion on every computed node: extra
 * nodes are pruned and missed splits refined, so the output equals mw_apply_batched's.  stats (may be
 * NULL): [0] triples, [1] passes, [2] proposed nodes, [3] pruned nodes, [4] refined misses,
 * [5] output nodes. */
int mw_apply_learned(int n, double prec, mw_tree* out, mw_op* ops, mw_tree* inp, int flags, mw_mlp mlp, float tau,
                     long long* stats);

#ifdef __cplusplus
}
#endif
#endif /* MWB200_H */
