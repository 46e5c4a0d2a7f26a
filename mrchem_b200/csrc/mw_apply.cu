// mw_apply.cu -- batched, adaptive NS-form apply on the device.
//
// A batch is any number of (output tree, operator, input tree) triples sharing one world (e.g. 32
// orbitals with 32 Helmholtz operators).  The refinement passes run in lock-step over the batch:
// pass d handles the depth-d output nodes of every tree with one launch per stage:
//   1. candidates: one warp per output node walks its operator's offset list, looks the input node
//      up in the input tree's hash index (or its leaf ancestor -> generated node) and screens it;
//   2. generated (scaling-only) input nodes are de-duplicated per tree and built once;
//   3. per candidate, the number of terms that pass the screening (the triples it contributes);
//   4. GEMM-tiled engine: the triples are expanded and sorted per output node by (term, dz, dy), and
//      each node's sorted triples are cut at plane boundaries into chunks of about chunk_triples
//      triples (a per-engine context setting, 48 unless tuned); the input blocks of the pass get
//      images in the kernel's staging layout.  Tensor-core and pencil engines: each node's candidate
//      list is cut into chunks of at most chunk_triples triples;
//   5. the contraction kernel runs one CTA per chunk; multi-chunk nodes write partial blocks that
//      a reduction kernel adds in chunk order (deterministic), single-chunk nodes write directly;
//   6. norms and split flags; children are appended to each tree.
// Results are identical to the per-node sequential order up to FP64 rounding.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <string>
#include <type_traits>

#include "mw_device.cuh"
#include "mw_kernels.cuh"
#include "mw_tmem.cuh"
#include "mw_umma.cuh"

namespace mwb {

constexpr double kTensorCoreMinPrec = 1e-6;  // finest prec served by the split-TF32 engine

struct BTree {
    const uint64_t* okey;
    double* ocoef;
    double* onorm2;
    double* ownorm2;
    InView in;
    const uint64_t* inkey;
    const DeltaRec* deltas;
    const TermRec* terms;
    const double* mats;
    const float* mats32;
    const double* matsb;    // beta-scaled copies (z-step operators)
    const float* matsb32;
    const double* matsT;    // transposed, zero-padded copies (GEMM-tiled contraction)
    const float* matsT32;
    const double* matsbT;
    const float* matsbT32;
    const float* matsI;  // split-TF32 operator images (tensor-core contraction)
    const float* matsbI;
    const float* matsS32;  // tensor-core x step engine: split-layout y/z operators and x-operator slices
    const float* matsbS32;
    const unsigned char* matsX;
    int nprefix;
    int root;
    double theta;
    double thr;  // split threshold of this pass
    int depth;   // depth of this entry's output nodes
    int depth_limit;
    long long ext[3];
    // block images of the pass (line-ordered contraction): input node i of this entry's depth has
    // image slot img_base + i - img_lb, for i in [img_lb, img_le)
    long long img_base;
    int img_lb, img_le;
};

struct Item {
    int tree;
    int node;
};

struct Chunk {
    int item;
    int c0, c1;
    int slot;  // partial block slot, -1: write the output node directly
};

// ---------------------------------------------------------------------------------------------
// 1. candidates
// ---------------------------------------------------------------------------------------------
__global__ void k_bcand(const Item* __restrict__ items, int nitems, const BTree* __restrict__ trees, int fill,
                        int* count, const int* offs, int* cdelta, int* csrc, uint64_t* greq_key, int* greq_leaf,
                        int* ngreq) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x & 31;
    if (w >= nitems) return;
    const Item it = items[w];
    const BTree& T = trees[it.tree];
    const int depth = T.depth;
    const long long ext[3] = {T.ext[0], T.ext[1], T.ext[2]};
    long long to[3];
    key_trans(T.okey[it.node], to);
    int kept = 0;
    const int base = fill ? offs[w] : 0;
    for (int b0 = 0; b0 < T.nprefix; b0 += 32) {
        const int e = b0 + lane;
        int ok = 0, src = 0, leaf = -1;
        uint64_t gk = kEmptyKey;
        if (e < T.nprefix) {
            const DeltaRec de = T.deltas[e];
            long long ti[3];
            bool inside = true;
            for (int d = 0; d < 3; ++d) {
                ti[d] = to[d] - de.d[d];
                if (ti[d] < 0 || ti[d] >= ext[d]) inside = false;
            }
            if (inside) {
                const uint64_t key = make_key(depth, ti[0], ti[1], ti[2]);
                const int idx = hlookup(T.in.hkey, T.in.hval, T.in.hcap, key);
                if (idx >= 0) {
                    const double nu = sqrt(T.in.norm2[idx]);
                    if (nu > 0.0 && de.maxb * nu >= T.theta) { ok = 1; src = idx; }
                } else {
                    for (int da = depth - 1; da >= 0 && leaf < 0; --da) {
                        const int sh = depth - da;
                        leaf = hlookup(T.in.hkey, T.in.hval, T.in.hcap, make_key(da, ti[0] >> sh, ti[1] >> sh, ti[2] >> sh));
                    }
                    const double nul = leaf >= 0 ? sqrt(T.in.norm2[leaf]) : 0.0;
                    if (nul > 0.0 && de.maxb * nul >= T.theta) {
                        ok = 1;
                        // entry index in place of the depth bits (an entry has one depth): unique
                        gk = ((uint64_t)it.tree << 57) | (key & ((1ull << 57) - 1));
                    }
                }
            }
        }
        const unsigned bal = __ballot_sync(0xffffffffu, ok);
        if (!fill) {  // the counting pass also counts the generated-node requests
            const unsigned gb = __ballot_sync(0xffffffffu, ok && gk != kEmptyKey);
            if (lane == 0 && gb) atomicAdd(ngreq, __popc(gb));
        }
        if (fill && ok) {
            const int pos = base + kept + __popc(bal & ((1u << lane) - 1u));
            cdelta[pos] = e;
            if (gk != kEmptyKey) {
                const int r = atomicAdd(ngreq, 1);
                greq_key[r] = gk;
                greq_leaf[r] = leaf;
                csrc[pos] = -(r + 1);
            } else {
                csrc[pos] = src;
            }
        }
        kept += __popc(bal);
    }
    if (!fill && lane == 0) count[w] = kept;
}

__global__ void k_bunique_flags(const uint64_t* __restrict__ k, int n, int* flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    flags[i] = (i == 0 || k[i] != k[i - 1]) ? 1 : 0;
}
__global__ void k_bunique_scatter(const uint64_t* __restrict__ k, const int* __restrict__ leaf,
                                  const int* __restrict__ flags, const int* __restrict__ pos, int n, uint64_t* uk,
                                  int* ul) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (flags[i]) {
        uk[pos[i]] = k[i];
        ul[pos[i]] = leaf[i];
    }
}
__global__ void k_bresolve_gen(int* csrc, int ncand, const uint64_t* __restrict__ greq_key,
                               const uint64_t* __restrict__ ukey, int nu) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ncand) return;
    const int s = csrc[i];
    if (s >= 0) return;
    const uint64_t key = greq_key[-s - 1];
    int lo = 0, hi = nu;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (ukey[mid] < key) lo = mid + 1; else hi = mid;
    }
    csrc[i] = -(lo + 1);
}

// ---------------------------------------------------------------------------------------------
// 2. generated input nodes: reconstruct the leaf ancestor, take the child on the path, descend
//    with zero wavelets (s_c = H_c^T s per dimension)
// ---------------------------------------------------------------------------------------------
// One direction of the two-scale reconstruction of a padded (2k)^3 shared block (out[o] = sum_i M[o][i]
// in[i], as pencil_transform) restricted to what child cc needs: outputs o in [cc[DIM] k, cc[DIM] k + k)
// only, on the pencils whose earlier directions' indices lie in the child's halves.
template <int K, int DIM>
__device__ static inline void child_transform(const double* __restrict__ M, double* A, const int (&cc)[3]) {
    using G = Geo<K>;
    constexpr int NPC = DIM == 0 ? G::K2 * G::K2 : DIM == 1 ? K * G::K2 : K * K;
    for (int p = threadIdx.x; p < NPC; p += blockDim.x) {
        int base, stride;
        if (DIM == 0) {  // all (y, z)
            base = G::P * ((p % G::K2) + G::K2 * (p / G::K2));
            stride = 1;
        } else if (DIM == 1) {  // x in the child's half, all z
            base = (cc[0] * K + p % K) + G::P * G::K2 * (p / K);
            stride = G::P;
        } else {  // x and y in the child's halves
            base = (cc[0] * K + p % K) + G::P * (cc[1] * K + p / K);
            stride = G::P * G::K2;
        }
        double x[G::K2];
#pragma unroll
        for (int i = 0; i < G::K2; ++i) x[i] = A[base + i * stride];
#pragma unroll 1
        for (int o = cc[DIM] * K; o < cc[DIM] * K + K; ++o) {
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < G::K2; ++i) s = fma(M[o * G::K2 + i], x[i], s);
            A[base + o * stride] = s;
        }
    }
}

template <int K>
__global__ void __launch_bounds__(256) k_bgenerate(const uint64_t* __restrict__ ukey, const int* __restrict__ uleaf,
                                                   const BTree* __restrict__ trees,
                                                   const double* __restrict__ FT, double* gblk, double* gnorm2) {
    using G = Geo<K>;
    extern __shared__ double sm[];
    double* A = sm;
    double* M = A + G::VOL;
    double* S = M + G::K2 * G::K2;
    double* red = S + K * K * K;
    const int g = blockIdx.x;
    const uint64_t gkey = ukey[g];
    const BTree& T = trees[(int)(gkey >> 57)];
    const int depth = T.depth;
    const int leaf = uleaf[g];
    for (int i = threadIdx.x; i < G::K2 * G::K2; i += blockDim.x) M[i] = FT[i];
    for (int e = threadIdx.x; e < G::BS; e += blockDim.x) {
        const int a = e % G::K2, b = (e / G::K2) % G::K2, c = e / (G::K2 * G::K2);
        A[G::at(a, b, c)] = T.in.coef[(size_t)leaf * G::BS + e];
    }
    long long t[3], tl[3];
    key_trans(gkey & ((1ull << 57) - 1), t);
    key_trans(T.inkey[leaf], tl);
    const int dl = depth - key_depth(T.inkey[leaf]);
    int cc[3];  // the leaf's child on the way down
    for (int q = 0; q < 3; ++q) cc[q] = (int)((t[q] >> (dl - 1)) - 2 * tl[q]);
    __syncthreads();
    // the leaf's reconstruction restricted to child cc: each direction computes only the outputs of the
    // child's half, over the inputs the next direction reads (same sums as the full transform)
    child_transform<K, 0>(M, A, cc);
    __syncthreads();
    child_transform<K, 1>(M, A, cc);
    __syncthreads();
    child_transform<K, 2>(M, A, cc);
    __syncthreads();
    for (int e = threadIdx.x; e < K * K * K; e += blockDim.x) {
        const int a = e % K, b = (e / K) % K, c = e / (K * K);
        S[e] = A[G::at(cc[0] * K + a, cc[1] * K + b, cc[2] * K + c)];
    }
    __syncthreads();
    for (int lev = dl - 2; lev >= 0; --lev) {
        for (int dim = 0; dim < 3; ++dim) {
            const int c = (int)((t[dim] >> lev) & 1);
            for (int p = threadIdx.x; p < K * K; p += blockDim.x) {
                const int u = p % K, v = p / K;
                int bs, st;
                if (dim == 0) { bs = K * (u + K * v); st = 1; }
                else if (dim == 1) { bs = u + K * K * v; st = K; }
                else { bs = u + K * v; st = K * K; }
                double x[K];
#pragma unroll
                for (int i = 0; i < K; ++i) x[i] = S[bs + i * st];
#pragma unroll 1
                for (int o = 0; o < K; ++o) {
                    double s = 0.0;
#pragma unroll
                    for (int i = 0; i < K; ++i) s = fma(M[(c * K + o) * G::K2 + i], x[i], s);
                    S[bs + o * st] = s;
                }
            }
            __syncthreads();
        }
    }
    double n2 = 0.0, dmy = 0.0;
    for (int e = threadIdx.x; e < K * K * K; e += blockDim.x) {
        const double v = S[e];
        gblk[(size_t)g * K * K * K + e] = v;
        n2 += v * v;
    }
    block_sum2(n2, dmy, red);
    if (threadIdx.x == 0) gnorm2[g] = n2;
}

// ---------------------------------------------------------------------------------------------
// 3-4. triples per candidate, chunks per output node
// ---------------------------------------------------------------------------------------------
__global__ void k_bterms(const int* __restrict__ cand_item, int ncand, const Item* __restrict__ items,
                         const BTree* __restrict__ trees, const int* __restrict__ cdelta, const int* __restrict__ csrc,
                         const double* __restrict__ gnorm2, int* ntrip) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ncand) return;
    const BTree& T = trees[items[cand_item[i]].tree];
    const int src = csrc[i];
    const double nu = src < 0 ? sqrt(gnorm2[-src - 1]) : sqrt(T.in.norm2[src]);
    const DeltaRec de = T.deltas[cdelta[i]];
    int n = 0;
    if (nu > 0.0 && !(de.maxb * nu < T.theta))
        for (int t = de.t0; t < de.t1 && !(T.terms[t].bound * nu < T.theta); ++t) ++n;
    ntrip[i] = n;
}
__global__ void k_cand_item(const int* __restrict__ offs, int nitems, int* cand_item) {
    const int w = blockIdx.x;
    if (w >= nitems) return;
    for (int c = offs[w] + threadIdx.x; c < offs[w + 1]; c += blockDim.x) cand_item[c] = w;
}
// greedy cut of each node's candidates into chunks of at most `limit` triples (whole
// candidates; at least one chunk per node so that every output block gets written)
__global__ void k_bchunks(const int* __restrict__ offs, int nitems, const int* __restrict__ ntrip, int limit, int fill,
                          int* nchunk, const int* __restrict__ choff, const int* __restrict__ slotoff, Chunk* chunks) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nitems) return;
    const int c0 = offs[w], c1 = offs[w + 1];
    int nch = 0, acc = 0, start = c0;
    const int multi = fill ? (choff[w + 1] - choff[w] > 1) : 0;
    for (int c = c0; c < c1; ++c) {
        const int t = ntrip[c];
        if (acc > 0 && acc + t > limit) {
            if (fill) chunks[choff[w] + nch] = Chunk{w, start, c, multi ? slotoff[w] + nch : -1};
            ++nch;
            acc = 0;
            start = c;
        }
        acc += t;
    }
    if (fill) chunks[choff[w] + nch] = Chunk{w, start, c1, multi ? slotoff[w] + nch : -1};
    ++nch;
    if (!fill) nchunk[w] = nch;
}
__global__ void k_multi_slots(const int* __restrict__ nchunk, int nitems, int* nslot) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nitems) return;
    nslot[w] = nchunk[w] > 1 ? nchunk[w] : 0;
}
// triples of the line-ordered contraction: candidate c contributes its first ntrip[c] term entries,
// at positions toff[c] ..; key = item << 32 | term << 20 | line rank (dz rank << 10 | dy rank),
// value = candidate << 32 | term entry.  A stable sort by key then groups every output node's
// triples by (term, dz, dy), in candidate order inside a line.
__global__ void k_texpand(const int* __restrict__ offs, const int* __restrict__ cand_item, int ncand, const Item* __restrict__ items,
                          const BTree* __restrict__ trees, const int* __restrict__ cdelta,
                          const int* __restrict__ ntrip, const int* __restrict__ toff,
                          const int* __restrict__ csrc, unsigned long long* key, unsigned long long* val, int* err) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncand) return;
    const int w = cand_item[c];
    const BTree& T = trees[items[w].tree];
    const DeltaRec de = T.deltas[cdelta[c]];
    const int n = ntrip[c], p0 = toff[c];
    const int src = csrc[c];
    if (n > 0 && src >= 0 && (src < T.img_lb || src >= T.img_le)) {  // not a node of this depth's level range
        atomicOr(err, 1);
        return;
    }
    // written mirrored inside the item's range, so that after the stable sort a line's triples come in
    // increasing order of their offset's bound (candidates are listed in decreasing order): the tensor
    // core's FP32 accumulation of a line's x sums rounds toward zero when it adds products of a smaller
    // scale to a larger sum, and adding the small contributions first loses fewer of their bits
    const int T0 = toff[offs[w]], T1 = toff[offs[w + 1]];
    for (int j = 0; j < n; ++j) {
        const int te = de.t0 + j;
        const int q = T0 + T1 - 1 - (p0 + j);
        key[q] = ((unsigned long long)w << 32) | ((unsigned long long)T.terms[te].m << 20) | (unsigned)de.lrank;
        val[q] = ((unsigned long long)c << 32) | (unsigned)te;
    }
}
// greedy cut of each node's sorted triples into chunks of about `limit` triples, at plane
// boundaries (a plane = the triples of one (term, dz); at least one chunk per node).  One warp per
// node: the plane starts of 32 triples at a time come from one ballot, and the cut walks the planes
// in order (a plane's size is known when the next one starts)
__global__ void k_tchunks(const int* __restrict__ offs, const int* __restrict__ toff, int nitems,
                          const unsigned long long* __restrict__ key, int limit, int fill, int* nchunk,
                          const int* __restrict__ choff, const int* __restrict__ slotoff, Chunk* chunks) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= nitems) return;  // uniform over the warp
    const int t0 = toff[offs[w]], t1 = toff[offs[w + 1]];
    int nch = 0, acc = 0, start = t0, ps = -1;  // ps: start of the plane being measured
    const int multi = fill ? (choff[w + 1] - choff[w] > 1) : 0;
    auto plane_done = [&](int end) {  // plane [ps, end) is complete: cut before it if it overflows
        const int sz = end - ps;
        if (acc > 0 && acc + sz > limit) {
            if (fill && lane == 0) chunks[choff[w] + nch] = Chunk{w, start, ps, multi ? slotoff[w] + nch : -1};
            ++nch;
            acc = 0;
            start = ps;
        }
        acc += sz;
    };
    for (int b = t0; b < t1; b += 32) {
        const int t = b + lane;
        bool st = false;
        if (t < t1)
            st = t == t0 ||
                 ((uint32_t)(key[t] & 0xffffffffull) >> 10) != ((uint32_t)(key[t - 1] & 0xffffffffull) >> 10);
        unsigned m = __ballot_sync(0xffffffffu, st);
        while (m) {
            const int p = b + __ffs(m) - 1;
            m &= m - 1;
            if (ps >= 0) plane_done(p);
            ps = p;
        }
    }
    if (ps >= 0) plane_done(t1);
    if (fill && lane == 0) chunks[choff[w] + nch] = Chunk{w, start, t1, multi ? slotoff[w] + nch : -1};
    ++nch;
    if (!fill && lane == 0) nchunk[w] = nch;
}
// Block images for the line-ordered contraction: image row a (a < 2k) holds X[a][b + P c] of the
// node block (P = 2k rounded up to 4; zero where b or c >= 2k), so that a CTA stages a block with
// 16-byte copies.  One CTA per block: read coalesced into shared memory, write the rows coalesced.
// Real nodes: entry e (a tree of the pass) contributes input nodes [lb[e], lb[e] + cnt[e]) at slots
// base[e] ..; generated nodes (k^3 scaling blocks) take slots gbase ...
struct ImgSrc {
    const double* coef;
    long long base;
    int lb, cnt;
};
template <int K, typename R>
__global__ void __launch_bounds__(256) k_ximage(const ImgSrc* __restrict__ srcs, int nsrc, const double* __restrict__ gblk,
                                                long long nreal, R* __restrict__ img) {
    constexpr int K2 = 2 * K, KP = (K2 + 3) / 4 * 4, NN = KP * KP, BS = K2 * K2 * K2, KKK = K * K * K;
    extern __shared__ __align__(16) unsigned char smraw[];
    R* blk = reinterpret_cast<R*>(smraw);
    const long long slot = blockIdx.x;
    if (slot < nreal) {
        int lo = 0, hi = nsrc - 1;  // last entry with base <= slot
        while (lo < hi) {
            const int mid = (lo + hi + 1) / 2;
            if (srcs[mid].base <= slot) lo = mid;
            else hi = mid - 1;
        }
        const ImgSrc sr = srcs[lo];
        const double* b = sr.coef + (size_t)(sr.lb + (slot - sr.base)) * BS;
        for (int e = threadIdx.x; e < BS; e += blockDim.x) blk[e] = (R)b[e];
    } else {
        const double* g = gblk + (size_t)(slot - nreal) * KKK;
        for (int e = threadIdx.x; e < BS; e += blockDim.x) {
            const int a = e % K2, bb = (e / K2) % K2, c = e / (K2 * K2);
            blk[e] = (a < K && bb < K && c < K) ? (R)g[a + K * (bb + K * c)] : R(0);
        }
    }
    __syncthreads();
    R* out = img + (size_t)slot * K2 * NN;
    for (int e = threadIdx.x; e < K2 * NN; e += blockDim.x) {
        const int a = e / NN, j = e - a * NN, b = j % KP, c = j / KP;
        out[e] = (b < K2 && c < K2) ? blk[a + K2 * (b + K2 * c)] : R(0);
    }
}

// ---------------------------------------------------------------------------------------------
// 5. contraction (one CTA per chunk), templated on the product type R:
//    R = double: the plain FP64 apply; R = float: FP32 products with FP64 accumulation of every
//    term's contribution (the mixed path).  Per term, three in-place pencil transforms:
//      out += beta (NS_z (x) NS_y (x) NS_x) in       out_sss -= beta (T_z (x) T_y (x) T_x) in_sss
//    (the second only at depth > 0: the s->s block belongs to coarser scales).
//    Each thread owns two pencils per step, so every operator element read from shared memory (as a
//    16-byte vector) feeds two FMA chains; the per-term matrices are double-buffered.
// ---------------------------------------------------------------------------------------------
template <typename R> struct VecT;
template <> struct VecT<double> { using T = double2; static constexpr int V = 2; };
template <> struct VecT<float> { using T = float4; static constexpr int V = 4; };

template <int K, typename R>
struct ACfg {
    static constexpr int K2 = 2 * K;
    static constexpr int NP = K2 * K2;
    static constexpr int LDM = (K2 + 3) / 4 * 4;          // padded operator row (16-byte vectors)
    static constexpr int MS = K2 * LDM;                     // one operator matrix
    static constexpr int P = K2 + 1;
    static constexpr int VOL = P * K2 * K2;                 // padded (2k)^3 tensor
    static constexpr bool STAGE = sizeof(R) * 2 * (size_t)VOL + sizeof(R) * 6 * MS <= 200 * 1024;
    static constexpr int XS = STAGE ? VOL : K * K * K;
    static constexpr int US = K * K * K;
    static constexpr int NT = ((NP / 2) + 31) / 32 * 32;    // two z-pencils per thread
    static constexpr size_t SMEM = sizeof(R) * (size_t)(XS + VOL + 6 * MS + US) + 64 * sizeof(double) + 64;
    __device__ static inline int at(int a, int b, int c) { return a + P * (b + K2 * c); }
};

// round n up to the vector width
template <typename R> __host__ __device__ constexpr int vround(int n) { return (n + VecT<R>::V - 1) / VecT<R>::V * VecT<R>::V; }

// out0[o] = sum_i M[o][i] x0[i], out1[o] = sum_i M[o][i] x1[i] for o < NOUT, i < NIN (x padded with
// zeros up to a multiple of the vector width)
template <typename R, int NIN, int LDM>
__device__ __forceinline__ void dot2(const R* __restrict__ Mrow, const R (&x0)[vround<R>(NIN)],
                                     const R (&x1)[vround<R>(NIN)], R& s0, R& s1) {
    using V = VecT<R>;
    s0 = R(0);
    s1 = R(0);
#pragma unroll
    for (int i = 0; i < vround<R>(NIN); i += V::V) {
        const typename V::T m = *reinterpret_cast<const typename V::T*>(Mrow + i);
        if constexpr (V::V == 2) {
            s0 = fma(m.x, x0[i], s0); s1 = fma(m.x, x1[i], s1);
            s0 = fma(m.y, x0[i + 1], s0); s1 = fma(m.y, x1[i + 1], s1);
        } else {
            s0 = fmaf(m.x, x0[i], s0); s1 = fmaf(m.x, x1[i], s1);
            s0 = fmaf(m.y, x0[i + 1], s0); s1 = fmaf(m.y, x1[i + 1], s1);
            s0 = fmaf(m.z, x0[i + 2], s0); s1 = fmaf(m.z, x1[i + 2], s1);
            s0 = fmaf(m.w, x0[i + 3], s0); s1 = fmaf(m.w, x1[i + 3], s1);
        }
    }
}

// generic pencil step over a padded shared tensor: for the pencils q of the step (two per
// thread iteration), y[o] = sum_i M[o][i] x[i], i < NIN, o < NOUT, in place (pencils are owned).
// base(q) / stride describe where a pencil lives.
template <int K, typename R, int NIN, int NOUT, int NPEN, typename BaseF>
__device__ __forceinline__ void pencil_step(const R* __restrict__ M, R* A, int stride, BaseF base) {
    using C = ACfg<K, R>;
    constexpr int NV = vround<R>(NIN);
    for (int q = 2 * threadIdx.x; q < NPEN; q += 2 * blockDim.x) {
        const bool two = q + 1 < NPEN;
        const int b0 = base(q), b1 = two ? base(q + 1) : b0;
        R x0[NV], x1[NV];
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            x0[i] = i < NIN ? A[b0 + i * stride] : R(0);
            x1[i] = i < NIN ? A[b1 + i * stride] : R(0);
        }
#pragma unroll 2
        for (int o = 0; o < NOUT; ++o) {
            R s0, s1;
            dot2<R, NIN, C::LDM>(M + o * C::LDM, x0, x1, s0, s1);
            A[b0 + o * stride] = s0;
            if (two) A[b1 + o * stride] = s1;
        }
    }
}

template <int K, typename R, bool GEN>
__device__ __forceinline__ void chain_xy(const R* Mx, const R* My, R* X, R* T, R* U, bool root, const double* blk,
                                         bool xfrom_global) {
    using C = ACfg<K, R>;
    constexpr int K2 = C::K2;
    constexpr int NIN = GEN ? K : K2;
    (void)blk;
    (void)xfrom_global;
    // x: T[:, b, c] = Mx X[:, b, c]   (pencils (b, c); GEN: b, c < k, inputs a < k)
    {
        constexpr int UX = GEN ? K : K2;
        constexpr int NV = vround<R>(NIN);
        for (int q = 2 * threadIdx.x; q < UX * UX; q += 2 * blockDim.x) {
            const bool two = q + 1 < UX * UX;
            const int bq0 = q % UX, cq0 = q / UX, bq1 = (q + 1) % UX, cq1 = (q + 1) / UX;
            R x0[NV], x1[NV];
#pragma unroll
            for (int i = 0; i < NV; ++i) {
                if (i < NIN) {
                    if (C::STAGE) {
                        x0[i] = X[C::at(i, bq0, cq0)];
                        x1[i] = two ? X[C::at(i, bq1, cq1)] : R(0);
                    } else if (GEN) {
                        x0[i] = X[i + K * (bq0 + K * cq0)];
                        x1[i] = two ? X[i + K * (bq1 + K * cq1)] : R(0);
                    } else {
                        x0[i] = (R)__ldg(&blk[i + K2 * (bq0 + K2 * cq0)]);
                        x1[i] = two ? (R)__ldg(&blk[i + K2 * (bq1 + K2 * cq1)]) : R(0);
                    }
                } else {
                    x0[i] = R(0);
                    x1[i] = R(0);
                }
            }
#pragma unroll 2
            for (int o = 0; o < K2; ++o) {
                R s0, s1;
                dot2<R, NIN, C::LDM>(Mx + o * C::LDM, x0, x1, s0, s1);
                T[C::at(o, bq0, cq0)] = s0;
                if (two) T[C::at(o, bq1, cq1)] = s1;
            }
        }
        if (!root) {
            constexpr int KV = vround<R>(K);
            for (int q = 2 * threadIdx.x; q < K * K; q += 2 * blockDim.x) {
                const bool two = q + 1 < K * K;
                const int bq0 = q % K, cq0 = q / K, bq1 = (q + 1) % K, cq1 = (q + 1) / K;
                R x0[KV], x1[KV];
#pragma unroll
                for (int i = 0; i < KV; ++i) {
                    if (i < K) {
                        if (C::STAGE) {
                            x0[i] = X[C::at(i, bq0, cq0)];
                            x1[i] = two ? X[C::at(i, bq1, cq1)] : R(0);
                        } else if (GEN) {
                            x0[i] = X[i + K * (bq0 + K * cq0)];
                            x1[i] = two ? X[i + K * (bq1 + K * cq1)] : R(0);
                        } else {
                            x0[i] = (R)__ldg(&blk[i + K2 * (bq0 + K2 * cq0)]);
                            x1[i] = two ? (R)__ldg(&blk[i + K2 * (bq1 + K2 * cq1)]) : R(0);
                        }
                    } else {
                        x0[i] = R(0);
                        x1[i] = R(0);
                    }
                }
#pragma unroll 2
                for (int o = 0; o < K; ++o) {
                    R s0, s1;
                    dot2<R, K, C::LDM>(Mx + o * C::LDM, x0, x1, s0, s1);
                    U[o + K * (bq0 + K * cq0)] = s0;
                    if (two) U[o + K * (bq1 + K * cq1)] = s1;
                }
            }
        }
    }
    __syncthreads();
    // y (in place): pencils (a, c), GEN: planes c < k, inputs b < k
    {
        constexpr int NC = GEN ? K : K2;
        pencil_step<K, R, NIN, K2, K2 * NC>(My, T, C::P, [](int q) { return ACfg<K, R>::at(q % (2 * K), 0, q / (2 * K)); });
        if (!root)
            pencil_step<K, R, K, K, K * K>(My, U, K, [](int q) { return (q % K) + K * K * (q / K); });
    }
}

template <int K, typename R>
__global__ void __launch_bounds__(ACfg<K, R>::NT, 1)
    k_bapply(const Chunk* __restrict__ chunks, const Item* __restrict__ items, const BTree* __restrict__ trees,
             const int* __restrict__ cdelta, const int* __restrict__ csrc, const double* __restrict__ gblk,
             const double* __restrict__ gnorm2, double* partials, unsigned long long* ntrip_out) {
    using C = ACfg<K, R>;
    constexpr int K2 = C::K2;
    constexpr int BS = K2 * K2 * K2;
    extern __shared__ __align__(16) unsigned char smraw[];
    R* X = reinterpret_cast<R*>(smraw);
    R* T = X + C::XS;
    R* Mb = T + C::VOL;  // [2][3][MS]
    R* U = Mb + 6 * C::MS;
    double* red = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(U + C::US) + 15) & ~uintptr_t(15));
    const Chunk ch = chunks[blockIdx.x];
    const Item it = items[ch.item];
    const BTree& TR = trees[it.tree];
    const R* mats = reinterpret_cast<const R*>(sizeof(R) == 8 ? (const void*)TR.mats : (const void*)TR.mats32);
    const bool root = TR.root != 0;
    const double theta = TR.theta;
    const int tid = threadIdx.x;
    double acc[2][K2];
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int c = 0; c < K2; ++c) acc[j][c] = 0.0;
    // the thread's two z-pencils (a, b)
    const int pz0 = 2 * tid, pz1 = 2 * tid + 1;
    const bool own0 = pz0 < C::NP, own1 = pz1 < C::NP;
    const int za0 = pz0 % K2, zb0 = pz0 / K2, za1 = pz1 % K2, zb1 = pz1 / K2;
    unsigned long long ntrip = 0;
    auto load_mats = [&](int buf, const TermRec& tr) {
        R* dst = Mb + buf * 3 * C::MS;
        for (int i = tid; i < 3 * C::MS; i += blockDim.x) {
            const int w = i / C::MS, r = (i % C::MS) / C::LDM, cc = (i % C::MS) % C::LDM;
            const int mi = w == 0 ? tr.mx : (w == 1 ? tr.my : tr.mz);
            dst[i] = cc < K2 ? mats[(size_t)mi * C::NP + r * K2 + cc] : R(0);
        }
    };
    for (int ci = ch.c0; ci < ch.c1; ++ci) {
        const int src = csrc[ci];
        const bool gen = src < 0;
        const double nu = gen ? sqrt(gnorm2[-src - 1]) : sqrt(TR.in.norm2[src]);
        const DeltaRec de = TR.deltas[cdelta[ci]];
        if (!(nu > 0.0) || de.maxb * nu < theta) continue;
        if (TR.terms[de.t0].bound * nu < theta) continue;
        const double* blk = gen ? gblk + (size_t)(-src - 1) * K * K * K : TR.in.coef + (size_t)src * BS;
        __syncthreads();  // previous candidate's users of X/T/U/M are done
        if (gen) {
            for (int e2 = tid; e2 < K * K * K; e2 += blockDim.x) {
                const int a = e2 % K, b = (e2 / K) % K, c = e2 / (K * K);
                if (C::STAGE) X[C::at(a, b, c)] = (R)blk[e2]; else X[e2] = (R)blk[e2];
            }
        } else if (C::STAGE) {
            for (int e2 = tid; e2 < BS; e2 += blockDim.x) {
                const int a = e2 % K2, b = (e2 / K2) % K2, c = e2 / (K2 * K2);
                X[C::at(a, b, c)] = (R)blk[e2];
            }
        }
        load_mats(0, TR.terms[de.t0]);
        int buf = 0;
        for (int ti = de.t0; ti < de.t1; ++ti) {
            const TermRec tr = TR.terms[ti];
            if (tr.bound * nu < theta) break;
            const R* Mx = Mb + buf * 3 * C::MS;
            const R* My = Mx + C::MS;
            const R* Mz = My + C::MS;
            __syncthreads();  // X, this term's matrices and the previous z-step are complete
            if (gen) chain_xy<K, R, true>(Mx, My, X, T, U, root, blk, !C::STAGE);
            else chain_xy<K, R, false>(Mx, My, X, T, U, root, blk, !C::STAGE);
            __syncthreads();
            // prefetch the next term's matrices into the other buffer while doing z
            if (ti + 1 < de.t1 && !(TR.terms[ti + 1].bound * nu < theta)) load_mats(buf ^ 1, TR.terms[ti + 1]);
            // z: acc[(a, b)][c'] += beta sum_c Mz[c'][c] T[a, b, c]
            {
                constexpr int NIN = K2;
                const int nin = gen ? K : K2;
                constexpr int NV = vround<R>(NIN);
                R x0[NV], x1[NV];
#pragma unroll
                for (int i = 0; i < NV; ++i) {
                    x0[i] = (own0 && i < nin) ? T[C::at(za0, zb0, i)] : R(0);
                    x1[i] = (own1 && i < nin) ? T[C::at(za1, zb1, i)] : R(0);
                }
#pragma unroll
                for (int o = 0; o < K2; ++o) {
                    R s0, s1;
                    dot2<R, NIN, C::LDM>(Mz + o * C::LDM, x0, x1, s0, s1);
                    acc[0][o] = fma(tr.beta, (double)s0, acc[0][o]);
                    acc[1][o] = fma(tr.beta, (double)s1, acc[1][o]);
                }
                if (!root) {
                    constexpr int KV = vround<R>(K);
                    const bool u0 = own0 && za0 < K && zb0 < K, u1 = own1 && za1 < K && zb1 < K;
                    if (u0 || u1) {
                        R y0[KV], y1[KV];
#pragma unroll
                        for (int i = 0; i < KV; ++i) {
                            y0[i] = (u0 && i < K) ? U[za0 + K * (zb0 + K * i)] : R(0);
                            y1[i] = (u1 && i < K) ? U[za1 + K * (zb1 + K * i)] : R(0);
                        }
#pragma unroll
                        for (int o = 0; o < K; ++o) {
                            R s0, s1;
                            dot2<R, K, C::LDM>(Mz + o * C::LDM, y0, y1, s0, s1);
                            if (u0) acc[0][o] = fma(-tr.beta, (double)s0, acc[0][o]);
                            if (u1) acc[1][o] = fma(-tr.beta, (double)s1, acc[1][o]);
                        }
                    }
                }
            }
            buf ^= 1;
            ++ntrip;
        }
    }
    double* dst = ch.slot < 0 ? TR.ocoef + (size_t)it.node * BS : partials + (size_t)ch.slot * BS;
    double n2 = 0.0, w2 = 0.0;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const bool own = j == 0 ? own0 : own1;
        const int a = j == 0 ? za0 : za1, b = j == 0 ? zb0 : zb1;
        if (own) {
#pragma unroll
            for (int c = 0; c < K2; ++c) {
                const double v = acc[j][c];
                dst[a + K2 * (b + K2 * c)] = v;
                n2 += v * v;
                if (!(a < K && b < K && c < K)) w2 += v * v;
            }
        }
    }
    block_sum2(n2, w2, red);
    if (tid == 0) {
        if (ch.slot < 0) {
            TR.onorm2[it.node] = n2;
            TR.ownorm2[it.node] = w2;
        }
        atomicAdd(ntrip_out, ntrip);
    }
}

// ---------------------------------------------------------------------------------------------
// 5b. GEMM-tiled contraction.  Each mode product of a term is a GEMM C[2k x (2k)^2] = M A with the
//     data operand in shared memory as k-major rows (row = contracted index, columns = the other two
//     indices), and every step writes its result in the row layout the next step reads:
//        X [a][b + P c]  --x-->  T1 [b][a' + P c]  --y-->  T2 [c][a' + P b']  --z-->  acc [c'][a' + P b']
//     (P = 2k rounded up to a multiple of 4, padding zero).  A thread owns an MT x NT tile of every
//     step; a warp is 4 row tiles x 8 column tiles, so per contracted index a warp reads MT broadcast
//     operator values and NT data values per lane and issues MT*NT FMAs.  Operators are staged
//     transposed (At[k][o] = M[o][k]); the z step uses the beta-scaled tables.
//     Below the root the s->s block is taken out with three k x k x k GEMMs on the top-left k x k
//     operator blocks (U1, U2, Uc); the owners of the z tiles subtract Uc one phase later.
//     Generated inputs (scaling part only) contract over k instead of 2k and skip the tiles that
//     only see their zero wavelet part.
//     Barriers per term: after x, after y.  Shared-memory hazards across terms are resolved by
//     loading each operator in a phase that the two barriers separate from its readers:
//     Mx(t+1) and Mz(t) during y(t), My(t+1) during z(t).
// ---------------------------------------------------------------------------------------------
__host__ __device__ constexpr int gcfg_nc(int k, int nthr) {
    int d = 1;
    while (d < k && (k % d != 0 || 2 * k * k / d > nthr)) ++d;
    return d;
}
// Row-stride padding of the T1 (x-step output) and T2 (y-step output) buffers, chosen per basis size
// so that the epilogue stores of a warp fall into few banks (counted wavefronts per step, consecutive
// column tiles per warp; the FP64 x step with an odd tile width uses strided tiles).  In FP32 the T1
// stride matches the 16-byte staging rows (T1 replaces a staged block at a line's end), which leaves
// two-way conflicts on the once-per-line T1 stores at k = 9, 10.
__host__ __device__ constexpr int gcfg_pad1(int k, bool f32) {
    return f32 ? ((k == 5 || k == 6 || k == 9 || k == 10 || k == 11 || k == 12) ? 4 : 0) : 0;
}
__host__ __device__ constexpr int gcfg_pad2(int k) {
    return (k == 5 || k == 6 || k == 9 || k == 10) ? 0 : (k == 11 || k == 12) ? 8 : 2;
}

template <int K, typename R>
struct GCfg {
    static constexpr bool F32 = sizeof(R) == 4;
    static constexpr int K2 = 2 * K;
    static constexpr int KP = (K2 + 3) / 4 * 4;
    static constexpr int NN = KP * KP;
    static constexpr int MT = KP / 4;
    static constexpr int NT = (F32 && MT * (KP / 2) <= 50) ? KP / 2 : KP / 4;
    static constexpr int LDX = NN + (F32 ? 4 : 2);  // 16-byte rows: staged by cp.async from the block images
    static constexpr int LD1 = NN + gcfg_pad1(K, F32);
    static constexpr int LD2 = NN + gcfg_pad2(K);
    static constexpr bool XSTRIDED = !F32 && (NT % 2 == 1);
    static constexpr int NTILE = NN / NT;
    static constexpr int NWARP = (NTILE + 7) / 8;
    static constexpr int NTHR = 32 * NWARP;
    static constexpr int KK = K * K;
    static constexpr int KKK = K * K * K;
    static constexpr int NC = gcfg_nc(K, NTHR);  // correction tile columns
    static constexpr int NCT = KK / NC;
    static constexpr int ND = MT * NT;  // accumulators per thread
    // FP32: accumulators in TMEM, 2 columns per double, warps sharing a lane quarter side by side
    static constexpr int TCOLS_NEED = ((NWARP + 3) / 4) * 2 * ND;
    static constexpr int TCOLS = TCOLS_NEED <= 32 ? 32 : TCOLS_NEED <= 64 ? 64 : TCOLS_NEED <= 128 ? 128
                                 : TCOLS_NEED <= 256 ? 256 : 512;
    static constexpr int XBUF = KP * (LDX > LD1 ? LDX : LD1);  // one staging buffer: X, or T1 at a line's end
    static constexpr int IMG = K2 * NN;                          // block image: rows a < 2k of X, unpadded
    static constexpr size_t SMEM =
        sizeof(R) * (2 * (size_t)XBUF + (size_t)KP * LD2 + 4 * (size_t)KP * KP + 3 * (size_t)KKK) + 64;
    static constexpr int MINB = (F32 && 2 * (SMEM + 16 + 1024) <= 233472) ? 2 : 1;
    static constexpr bool FITS = SMEM + 16 + 1024 <= 232448 && 2 * NCT <= NTHR && TCOLS_NEED <= 512 &&
                                 (size_t)KP * LDX * sizeof(R) >= 64 * sizeof(double) && (!F32 || TCOLS * MINB <= 512);
};

__device__ __forceinline__ float mfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double mfma(double a, double b, double c) { return fma(a, b, c); }

// packed FP32 pairs (sm_100 f32x2 arithmetic): two independent round-to-nearest FMAs per instruction,
// bit-identical to two fmaf calls
__device__ __forceinline__ unsigned long long fma_f32x2(unsigned long long a, unsigned long long b,
                                                        unsigned long long c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ unsigned long long pack_f32x2(float lo, float hi) {
    unsigned long long d;
    asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(lo), "f"(hi));
    return d;
}
__device__ __forceinline__ void unpack_f32x2(unsigned long long v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}

// c (+)= At^T B on a thread tile: c[i][j] (+)= sum_{k < kdim} At[k lda + o0 + i] B[k ldb + n0 + j]
template <int MT, int NT, bool ACC, typename R, typename CT>
__device__ __forceinline__ void gemm_tile(const R* __restrict__ At, int lda, const R* __restrict__ B, int ldb,
                                          int o0, int n0, int kdim, CT (&c)[MT][NT]) {
    if constexpr (sizeof(R) == 4 && sizeof(CT) == 4 && NT % 2 == 0) {
        // FP32 tile: column pairs in packed registers, one f32x2 FMA per pair and contracted index
        constexpr int NP = NT / 2;
        unsigned long long pc[MT][NP];
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < NP; ++j) pc[i][j] = ACC ? pack_f32x2(c[i][2 * j], c[i][2 * j + 1]) : 0ull;
        const R* ap = At + o0;
        const R* bp = B + n0;
#pragma unroll 2
        for (int k = 0; k < kdim; ++k) {
            unsigned long long a2[MT], b2[NP];
#pragma unroll
            for (int i = 0; i < MT; ++i) a2[i] = pack_f32x2(ap[i], ap[i]);
#pragma unroll
            for (int j = 0; j < NP; ++j) b2[j] = *reinterpret_cast<const unsigned long long*>(bp + 2 * j);
#pragma unroll
            for (int i = 0; i < MT; ++i)
#pragma unroll
                for (int j = 0; j < NP; ++j) pc[i][j] = fma_f32x2(a2[i], b2[j], pc[i][j]);
            ap += lda;
            bp += ldb;
        }
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < NP; ++j) unpack_f32x2(pc[i][j], c[i][2 * j], c[i][2 * j + 1]);
        return;
    }
    if (!ACC) {
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < NT; ++j) c[i][j] = CT(0);
    }
    const R* ap = At + o0;
    const R* bp = B + n0;
#pragma unroll 2
    for (int k = 0; k < kdim; ++k) {
        R a[MT], b[NT];
#pragma unroll
        for (int i = 0; i < MT; ++i) a[i] = ap[i];
        if constexpr (NT % 2 == 0) {
            using V2 = typename std::conditional<sizeof(R) == 4, float2, double2>::type;
#pragma unroll
            for (int j = 0; j < NT; j += 2) {
                const V2 v = *reinterpret_cast<const V2*>(bp + j);
                b[j] = v.x;
                b[j + 1] = v.y;
            }
        } else {
#pragma unroll
            for (int j = 0; j < NT; ++j) b[j] = bp[j];
        }
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < NT; ++j) c[i][j] = mfma((CT)a[i], (CT)b[j], c[i][j]);
        ap += lda;
        bp += ldb;
    }
}

// FP32 tile with packed accumulators kept across calls: pc[i][j] (+)= sum_k At[k lda + o0 + i] times the
// column pair B[k ldb + n0 + 2j], B[k ldb + n0 + 2j + 1] (the same FMAs as gemm_tile's FP32 path)
template <int MT, int NP>
__device__ __forceinline__ void gemm_tile_packed(const float* __restrict__ At, int lda, const float* __restrict__ B,
                                                 int ldb, int o0, int n0, int kdim, unsigned long long (&pc)[MT][NP]) {
    const float* ap = At + o0;
    const float* bp = B + n0;
#pragma unroll 2
    for (int k = 0; k < kdim; ++k) {
        unsigned long long a2[MT], b2[NP];
#pragma unroll
        for (int i = 0; i < MT; ++i) a2[i] = pack_f32x2(ap[i], ap[i]);
#pragma unroll
        for (int j = 0; j < NP; ++j) b2[j] = *reinterpret_cast<const unsigned long long*>(bp + 2 * j);
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < NP; ++j) pc[i][j] = fma_f32x2(a2[i], b2[j], pc[i][j]);
        ap += lda;
        bp += ldb;
    }
}

// the same with per-column offsets (correction GEMMs; columns not contiguous)
template <int MT, int NT, typename R>
__device__ __forceinline__ void gemm_tile_off(const R* __restrict__ At, int lda, const R* __restrict__ B, int ldb,
                                              int o0, const int (&off)[NT], int kdim, R (&c)[MT][NT]) {
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j) c[i][j] = R(0);
    for (int k = 0; k < kdim; ++k) {
        R a[MT], b[NT];
#pragma unroll
        for (int i = 0; i < MT; ++i) a[i] = At[k * lda + o0 + i];
#pragma unroll
        for (int j = 0; j < NT; ++j) b[j] = B[k * ldb + off[j]];
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < NT; ++j) c[i][j] = mfma(a[i], b[j], c[i][j]);
    }
}

// Line-ordered GEMM-tiled contraction.  A chunk is a range of one output node's surviving triples,
// sorted by (term, dz, dy): a *line* is a run of triples with the same (term, dz, dy) and a *plane* a
// run with the same (term, dz).  Because a term's operator is separable,
//   sum_l  Mz(dz) My(dy) Mx(dx) in_l  =  sum_dz Mz(dz) [ sum_dy My(dy) [ sum_dx Mx(dx) in_l ] ],
// so every triple costs one x mode product (summed over its line in registers), every line one y mode
// product (summed over its plane in T2) and every plane one z mode product (summed into the output
// block), instead of three mode products per triple.  The s->s correction below the root follows the
// same grouping on its k^3 blocks.
// Input blocks are staged from their images (the X layout in `R`, built per pass) into two buffers
// by cp.async: the next triple's block and operator load while the current triple computes.  At a
// line's end its x sums (T1) replace the line's last block in its buffer.
// tkey (sorted): item << 32 | term << 20 | dz rank << 10 | dy rank; tval: candidate << 32 | term entry.
template <int K, typename R>
__global__ void __launch_bounds__(GCfg<K, R>::NTHR, GCfg<K, R>::MINB)
    k_gapply(const Chunk* __restrict__ chunks, const Item* __restrict__ items, const BTree* __restrict__ trees,
             const unsigned long long* __restrict__ tkey, const unsigned long long* __restrict__ tval,
             const int* __restrict__ csrc, const R* __restrict__ ximg, long long gbase, double* partials,
             unsigned long long* ntrip_out) {
    using C = GCfg<K, R>;
    constexpr int K2 = C::K2, KP = C::KP, MT = C::MT, NT = C::NT, NC = C::NC, ND = C::ND;
    constexpr int LDX = C::LDX, LD1 = C::LD1, LD2 = C::LD2, NN = C::NN, IMG = C::IMG;
    constexpr int KK = C::KK, KKK = C::KKK;
    constexpr int BS = K2 * K2 * K2;
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ uint32_t tmem_slot;
    R* XA = reinterpret_cast<R*>(smraw);  // staging buffers: X [KP][LDX], or T1 [KP][LD1]
    R* XB = XA + C::XBUF;
    R* T2 = XB + C::XBUF;                 // [KP][LD2]
    R* Mx0 = T2 + KP * LD2;               // [KP][KP], At[k][o] = M[o][k]; x operators of the two buffers
    R* Mx1 = Mx0 + KP * KP;
    R* My = Mx1 + KP * KP;
    R* Mz = My + KP * KP;
    R* U1 = Mz + KP * KP;  // [K][K][K]
    R* U2 = U1 + KKK;
    R* Uc = U2 + KKK;
    const Chunk ch = chunks[blockIdx.x];
    const Item it = items[ch.item];
    const BTree& TR = trees[it.tree];
    const R* mats = reinterpret_cast<const R*>(C::F32 ? (const void*)TR.matsT32 : (const void*)TR.matsT);
    const R* matsb = reinterpret_cast<const R*>(C::F32 ? (const void*)TR.matsbT32 : (const void*)TR.matsbT);
    const bool root = TR.root != 0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // tiles: 4 row tiles x 8 column tiles per warp; consecutive column tiles (y and z steps, and the
    // x step unless strided), or column tiles strided by the warp count (x step)
    const int rt = lane & 3;
    const int ct_c = warp * 8 + (lane >> 2);
    const int ct_x = C::XSTRIDED ? warp + C::NWARP * (lane >> 2) : ct_c;
    const bool own = ct_c < C::NTILE, own_x = ct_x < C::NTILE;
    const int o0 = rt * MT;
    const int n0 = own ? ct_c * NT : 0, n0x = own_x ? ct_x * NT : 0;
    const int tb0 = n0 % KP, tc0 = n0 / KP;     // y tile: first a', c;  z tile: first a', b'
    const int xb0 = n0x % KP, xc0 = n0x / KP;   // x tile: first b, c
    // correction tile
    const int crt = tid & 1, cct = tid >> 1;
    const bool cown = !root && cct < C::NCT;
    const int co0 = crt * MT, cn0 = cown ? cct * NC : 0;

    // accumulators: registers (FP64 kernel) or this thread's TMEM lane (FP32 kernel)
    double acc[C::F32 ? 1 : MT][C::F32 ? 1 : NT];
    uint32_t tacc = 0;
    if constexpr (C::F32) {
        if (warp == 0) {
            tmem_alloc(&tmem_slot, C::TCOLS);
            tmem_relinquish();
        }
        tmem_fence_before_sync();
        __syncthreads();
        tmem_fence_after_sync();
        tacc = tmem_slot + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)((warp >> 2) * 2 * ND);
        tmem_visit<ND, true>(tacc, [&](int, int n, auto& r) {
#pragma unroll
            for (int q = 0; q < 2 * n; ++q) r[q] = 0u;
        });
    } else {
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < NT; ++j) acc[i][j] = 0.0;
    }
    unsigned long long ntrip = 0;
    bool pend2 = false;     // c2 holds a correction block not yet written to Uc
    bool uc_valid = false;  // Uc holds a correction block not yet subtracted
    R c2[MT][NC];
    // x sums of the current line (this thread's x tile): FP32 column pairs packed (f32x2), or plain
    constexpr bool PK = C::F32 && NT % 2 == 0;
    unsigned long long xp[PK ? MT : 1][PK ? NT / 2 : 1];
    R xacc[PK ? 1 : MT][PK ? 1 : NT];

    // asynchronous copy of a transposed operator (At[k][o] = M[o][k], P x P) into shared memory, as
    // one commit group
    auto load_mat = [&](R* dst, const R* tab, int mi) {
        constexpr int NV = KP * KP * (int)sizeof(R) / 16;
        const char* src = reinterpret_cast<const char*>(tab + (size_t)mi * KP * KP);
        for (int e = tid; e < NV; e += blockDim.x) cp_async16(reinterpret_cast<char*>(dst) + 16 * e, src + 16 * e);
        cp_async_commit();
    };
    auto image_of = [&](int t) -> const R* {
        const int src = csrc[(int)(tval[t] >> 32)];
        const long long slot = src < 0 ? gbase + (-src - 1) : TR.img_base + (src - TR.img_lb);
        return ximg + (size_t)slot * IMG;
    };
    // triple t's block image into buffer q (rows a < 2k; the rows of X beyond are never read) and its
    // x operator, one commit group
    auto stage = [&](int t, int q) {
        const R* img = image_of(t);
        R* dst = q ? XB : XA;
        constexpr int RV = NN * (int)sizeof(R) / 16;  // 16-byte vectors per row
        constexpr int EV = 16 / (int)sizeof(R);
        for (int e = tid; e < K2 * RV; e += blockDim.x) {
            const int a = e / RV, v = e - a * RV;
            cp_async16(dst + a * LDX + v * EV, img + (size_t)a * NN + v * EV);
        }
        load_mat(q ? Mx1 : Mx0, mats, TR.terms[(int)(tval[t] & 0xffffffffull)].mx);
    };
    // correction block of element (c', a', b') of this thread's z tile, 0 outside s->s
    auto uc_at = [&](int i, int j) -> double {
        const int cz = o0 + i, n = n0 + j, ax = n % KP, by = n / KP;
        return (cz < K && ax < K && by < K) ? (double)Uc[cz * KK + ax + K * by] : 0.0;
    };
    auto write_c2 = [&]() {
        if (!cown) return;
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < NC; ++j)
                if (co0 + i < K) Uc[(co0 + i) * KK + cn0 + j] = c2[i][j];
    };

    auto line_of = [&](int t) -> uint32_t { return (uint32_t)(tkey[t] & 0xffffffffull); };
    bool line_gen = true;    // every triple of the current line has a generated (scaling-only) input
    bool plane_gen = true;   // ... of the current plane
    bool first_line = true;  // the current line is the first of its plane
    if (ch.c0 < ch.c1) stage(ch.c0, 0);
    int q = 0;  // buffer of the current triple
    for (int t = ch.c0; t < ch.c1; ++t, q ^= 1) {
        const unsigned long long tv = tval[t];
        const bool gen = csrc[(int)(tv >> 32)] < 0;
        const TermRec tr = TR.terms[(int)(tv & 0xffffffffull)];
        const uint32_t lk = line_of(t);
        const bool lstart = t == ch.c0 || line_of(t - 1) != lk;
        const bool pstart = t == ch.c0 || (line_of(t - 1) >> 10) != (lk >> 10);
        const bool lend = t + 1 == ch.c1 || line_of(t + 1) != lk;
        const bool pend = t + 1 == ch.c1 || (line_of(t + 1) >> 10) != (lk >> 10);
        const bool more = t + 1 < ch.c1;
        if (pstart) {
            plane_gen = true;
            first_line = true;
        }
        if (lstart) line_gen = true;
        line_gen = line_gen && gen;
        plane_gen = plane_gen && gen;
        cp_async_wait_all();
        __syncthreads();  // triple t's block and x operator are in; every reader of the other buffer, of
                          // My, Mz, T2, U1, U2 and Uc from earlier steps is done
        if (lend) load_mat(My, mats, tr.my);
        if (pend) load_mat(Mz, matsb, tr.mz);
        if (more) stage(t + 1, q ^ 1);
        if (tid == 0 && t + 2 < ch.c1) prefetch_l2_bulk(image_of(t + 2), (unsigned)(IMG * sizeof(R)));
        R* Xq = q ? XB : XA;
        const R* Mxq = q ? Mx1 : Mx0;
        // ---- x: xacc[a'][b + P c] (+)= sum_a Mx[a'][a] X[a][b + P c]   (a line sums its triples)
        if (own_x) {
            const bool live = !gen || (xb0 < K && xc0 < K);  // other tiles of a generated input are zero
            if constexpr (PK) {
                if (lstart) {
#pragma unroll
                    for (int i = 0; i < MT; ++i)
#pragma unroll
                        for (int j = 0; j < NT / 2; ++j) xp[i][j] = 0ull;
                }
                if (live)
                    gemm_tile_packed<MT, NT / 2>(reinterpret_cast<const float*>(Mxq), KP,
                                                 reinterpret_cast<const float*>(Xq), LDX, o0, n0x, gen ? K : K2, xp);
            } else {
                if (lstart) {
#pragma unroll
                    for (int i = 0; i < MT; ++i)
#pragma unroll
                        for (int j = 0; j < NT; ++j) xacc[i][j] = R(0);
                }
                if (live) gemm_tile<MT, NT, true>(Mxq, KP, Xq, LDX, o0, n0x, gen ? K : K2, xacc);
            }
        }
        if (cown) {  // U1[b][a' + k c] (+)= sum_{a<k} Tx[a'][a] X[a][b + P c]   (summed over the line)
            int off[NC];
#pragma unroll
            for (int j = 0; j < NC; ++j) off[j] = (cn0 + j) % K + KP * ((cn0 + j) / K);
            R c[MT][NC];
            gemm_tile_off<MT, NC>(Mxq, KP, Xq, LDX, co0, off, K, c);
#pragma unroll
            for (int i = 0; i < MT; ++i)
#pragma unroll
                for (int j = 0; j < NC; ++j) {
                    const int n = cn0 + j;
                    if (co0 + i < K) {
                        R& d = U1[(n % K) * KK + co0 + i + K * (n / K)];
                        d = lstart ? c[i][j] : d + c[i][j];
                    }
                }
        }
        ++ntrip;
        if (!lend) continue;
        __syncthreads();  // every reader of Xq is done: the line's x sums replace its last block
        R* T1 = Xq;       // [KP][LD1]
        if (own_x) {
            if constexpr (PK) {
#pragma unroll
                for (int j = 0; j < NT / 2; ++j)
#pragma unroll
                    for (int i = 0; i < MT; ++i) {
                        float lo, hi;
                        unpack_f32x2(xp[i][j], lo, hi);
                        T1[(xb0 + 2 * j) * LD1 + o0 + i + KP * xc0] = lo;
                        T1[(xb0 + 2 * j + 1) * LD1 + o0 + i + KP * xc0] = hi;
                    }
            } else {
#pragma unroll
                for (int j = 0; j < NT; ++j)
#pragma unroll
                    for (int i = 0; i < MT; ++i) T1[(xb0 + j) * LD1 + o0 + i + KP * xc0] = xacc[i][j];
            }
        }
        // My (and Mz) were committed before the next triple's staging group
        if (more) cp_async_wait_group<1>();
        else cp_async_wait_all();
        __syncthreads();  // T1, U1, My and Mz are in
        // ---- y: T2[c][a' + P b'] (+)= sum_b My[b'][b] T1[b][a' + P c]   (a plane sums its lines)
        if (pend2) {  // the previous plane's correction block, subtracted in this plane's z phase
            write_c2();
            pend2 = false;
            uc_valid = true;
        }
        if (own) {
            const bool zero = line_gen && !(tc0 < K);  // this tile is zero for generated inputs
            if (!zero || first_line) {
                R c[MT][NT];
                if (zero) {
#pragma unroll
                    for (int i = 0; i < MT; ++i)
#pragma unroll
                        for (int j = 0; j < NT; ++j) c[i][j] = R(0);
                } else {
                    gemm_tile<MT, NT, false>(My, KP, T1, LD1, o0, n0, line_gen ? K : K2, c);
                }
#pragma unroll
                for (int i = 0; i < MT; ++i) {
                    R* row = T2 + tc0 * LD2 + tb0 + KP * (o0 + i);
                    if constexpr (NT % 2 == 0) {
                        using V2 = typename std::conditional<sizeof(R) == 4, float2, double2>::type;
#pragma unroll
                        for (int j = 0; j < NT; j += 2) {
                            V2 v;
                            if (first_line) {
                                v.x = c[i][j];
                                v.y = c[i][j + 1];
                            } else {
                                v = *reinterpret_cast<const V2*>(row + j);
                                v.x += c[i][j];
                                v.y += c[i][j + 1];
                            }
                            *reinterpret_cast<V2*>(row + j) = v;
                        }
                    } else {
#pragma unroll
                        for (int j = 0; j < NT; ++j) row[j] = first_line ? c[i][j] : row[j] + c[i][j];
                    }
                }
            }
        }
        if (cown) {  // U2[c][a' + k b'] (+)= sum_{b<k} Ty[b'][b] U1[b][a' + k c]
            int off[NC];
#pragma unroll
            for (int j = 0; j < NC; ++j) off[j] = cn0 + j;
            R c[MT][NC];
            gemm_tile_off<MT, NC>(My, KP, U1, KK, co0, off, K, c);
#pragma unroll
            for (int i = 0; i < MT; ++i)
#pragma unroll
                for (int j = 0; j < NC; ++j) {
                    const int n = cn0 + j;
                    if (co0 + i < K) {
                        R& d = U2[(n / K) * KK + (n % K) + K * (co0 + i)];
                        d = first_line ? c[i][j] : d + c[i][j];
                    }
                }
        }
        first_line = false;
        if (!pend) continue;
        __syncthreads();  // T2, U2 and Uc of the plane are complete
        // ---- z: acc[c'][a' + P b'] += sum_c (beta Mz)[c'][c] T2[c][a' + P b']  (- previous correction)
        const int kdz = plane_gen ? K : K2;
        if constexpr (C::F32) {
            float c[MT][NT];
            if (own) {
                gemm_tile<MT, NT, false>(Mz, KP, T2, LD2, o0, n0, kdz, c);
            } else {
#pragma unroll
                for (int i = 0; i < MT; ++i)
#pragma unroll
                    for (int j = 0; j < NT; ++j) c[i][j] = 0.0f;
            }
            const bool fold = uc_valid && own;
            tmem_visit<ND, true>(tacc, [&](int d0, int n, auto& r) {
#pragma unroll
                for (int q2 = 0; q2 < n; ++q2) {
                    const int d = d0 + q2, i = d / NT, j = d % NT;
                    double v = words_to_double(r[2 * q2], r[2 * q2 + 1]) + (double)c[i][j];
                    if (fold) v -= uc_at(i, j);
                    double_to_words(v, r[2 * q2], r[2 * q2 + 1]);
                }
            });
        } else {
            if (own) {
                gemm_tile<MT, NT, true>(Mz, KP, T2, LD2, o0, n0, kdz, acc);
                if (uc_valid) {
#pragma unroll
                    for (int i = 0; i < MT; ++i)
#pragma unroll
                        for (int j = 0; j < NT; ++j) acc[i][j] -= uc_at(i, j);
                }
            }
        }
        uc_valid = false;
        if (cown) {  // c2[c'][a' + k b'] = sum_{c<k} (beta Tz)[c'][c] U2[c][a' + k b']
            int off[NC];
#pragma unroll
            for (int j = 0; j < NC; ++j) off[j] = cn0 + j;
            gemm_tile_off<MT, NC>(Mz, KP, U2, KK, co0, off, K, c2);
        }
        pend2 = !root;
    }
    cp_async_wait_all();
    __syncthreads();  // z-phase readers of Uc are done
    if (pend2) write_c2();
    uc_valid = pend2;
    __syncthreads();
    double* dst = ch.slot < 0 ? TR.ocoef + (size_t)it.node * BS : partials + (size_t)ch.slot * BS;
    double n2 = 0.0, w2 = 0.0;
    auto emit = [&](int i, int j, double v) {
        const int cz = o0 + i, n = n0 + j, ax = n % KP, by = n / KP;
        if (uc_valid) v -= uc_at(i, j);
        if (cz < K2 && ax < K2 && by < K2) {
            dst[ax + K2 * (by + K2 * cz)] = v;
            n2 += v * v;
            if (!(ax < K && by < K && cz < K)) w2 += v * v;
        }
    };
    if constexpr (C::F32) {
        tmem_visit<ND, false>(tacc, [&](int d0, int n, auto& r) {
#pragma unroll
            for (int q = 0; q < n; ++q) {
                const int d = d0 + q;
                if (own) emit(d / NT, d % NT, words_to_double(r[2 * q], r[2 * q + 1]));
            }
        });
        tmem_fence_before_sync();
        __syncthreads();
        tmem_fence_after_sync();
        if (warp == 0) tmem_dealloc(tmem_slot, C::TCOLS);
    } else {
        if (own) {
#pragma unroll
            for (int i = 0; i < MT; ++i)
#pragma unroll
                for (int j = 0; j < NT; ++j) emit(i, j, acc[i][j]);
        }
    }
    double* red = reinterpret_cast<double*>(XA);  // the staging buffers are no longer read
    __syncthreads();
    block_sum2(n2, w2, red);
    if (tid == 0) {
        if (ch.slot < 0) {
            TR.onorm2[it.node] = n2;
            TR.ownorm2[it.node] = w2;
        }
        atomicAdd(ntrip_out, ntrip);
    }
}

}  // namespace mwb
#include "mw_tapply.cuh"
#include "mw_happly.cuh"
namespace mwb {

// triples of every chunk (the sort key of the longest-first launch order); chunks never exceed 2^16 triples
__global__ void k_chunk_len(const Chunk* __restrict__ chunks, int n, int* __restrict__ len) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) len[i] = min(chunks[i].c1 - chunks[i].c0, 65535);
}

// add the partial blocks of a multi-chunk node in chunk order; write block and norms
template <int K>
__global__ void __launch_bounds__(256) k_breduce(const Chunk* __restrict__ chunks, const int* __restrict__ choff,
                                                 const int* __restrict__ multi_items, const Item* __restrict__ items,
                                                 const BTree* __restrict__ trees, const double* __restrict__ partials) {
    using G = Geo<K>;
    __shared__ double red[64];
    const int w = multi_items ? multi_items[blockIdx.x] : blockIdx.x;  // no list: one block per item
    const int cb = choff[w], ce = choff[w + 1];
    if (ce - cb < 2) return;  // a single chunk wrote the node itself
    const Item it = items[w];
    const BTree& TR = trees[it.tree];
    double n2 = 0.0, w2 = 0.0;
    for (int e = threadIdx.x; e < G::BS; e += blockDim.x) {
        double v = 0.0;
        for (int c = cb; c < ce; ++c) v += partials[(size_t)chunks[c].slot * G::BS + e];
        TR.ocoef[(size_t)it.node * G::BS + e] = v;
        const int a = e % G::K2, b = (e / G::K2) % G::K2, cc = e / (G::K2 * G::K2);
        n2 += v * v;
        if (!(a < K && b < K && cc < K)) w2 += v * v;
    }
    block_sum2(n2, w2, red);
    if (threadIdx.x == 0) {
        TR.onorm2[it.node] = n2;
        TR.ownorm2[it.node] = w2;
    }
}

// ---------------------------------------------------------------------------------------------
// 6. per-tree root norms, split flags
// ---------------------------------------------------------------------------------------------
__global__ void k_tree_item_norm2(const Item* __restrict__ items, const int* __restrict__ item_off,
                                  const BTree* __restrict__ trees, double* out) {
    __shared__ double red[64];
    const int t = blockIdx.x;
    double s = 0.0, d = 0.0;
    for (int i = item_off[t] + threadIdx.x; i < item_off[t + 1]; i += blockDim.x) s += trees[t].onorm2[items[i].node];
    block_sum2(s, d, red);
    if (threadIdx.x == 0) out[t] = s;
}
// split thresholds of the root entries from their output norms: prec g0 with g0 the square root of the
// root level's square norm (the same operations as the host's prec g0 2^(-depth/2) at depth 0)
__global__ void k_root_thr(BTree* trees, const double* __restrict__ g, const double* __restrict__ prec, int nt) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt || trees[t].depth != 0) return;
    const double g0 = sqrt(g[t]);
    trees[t].thr = (prec[t] > 0.0 && g0 > 0.0) ? prec[t] * g0 : INFINITY;
}
__global__ void k_bsplit_flags(const Item* __restrict__ items, int nitems, const BTree* __restrict__ trees,
                               int* flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nitems) return;
    const Item it = items[i];
    const BTree& T = trees[it.tree];
    flags[i] = (T.depth < T.depth_limit && sqrt(T.ownorm2[it.node]) > T.thr) ? 1 : 0;
}

// ---------------------------------------------------------------------------------------------
// driver
// ---------------------------------------------------------------------------------------------

static inline void count(Ctx* c, int n = 1) { c->launches += n; }

// MWB200_CONTRACTION=pencil selects the pencil contraction kernel even where the GEMM-tiled one fits
// (both compute the same sums; kept for comparison and for bases too large for the tiled kernel)
static bool contraction_pencil() {
    static const bool v = [] {
        const char* e = std::getenv("MWB200_CONTRACTION");
        return e != nullptr && std::string(e) == "pencil";
    }();
    return v;
}

template <typename T>
static T* upload(Ctx* ctx, const std::vector<T>& v) {
    T* d = (T*)dalloc(ctx, sizeof(T) * std::max<size_t>(1, v.size()));
    upload_bytes(ctx, d, v.data(), sizeof(T) * v.size());
    return d;
}
// exclusive sum of d_in[0 .. n] into d_out (the total lands in d_out[n]); no host read-back
static void scan_only(Ctx* ctx, const int* d_in, int* d_out, int n) {
    size_t tmp = 0;
    MWB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, d_in, d_out, n + 1, ctx->stream));
    void* d_tmp = dalloc(ctx, tmp);
    MWB_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp, tmp, d_in, d_out, n + 1, ctx->stream));
    dfree(ctx, d_tmp);
}
static int scan_total(Ctx* ctx, const int* d_in, int* d_out, int n) {
    size_t tmp = 0;
    MWB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, d_in, d_out, n + 1, ctx->stream));
    void* d_tmp = dalloc(ctx, tmp);
    MWB_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp, tmp, d_in, d_out, n + 1, ctx->stream));
    dfree(ctx, d_tmp);
    int total = 0;
    readback(ctx, {{&total, d_out + n, sizeof(int)}});
    return total;
}

#define MWB_DISPATCH_K(k, F)                                             \
    switch (k) {                                                         \
        case 4: F(4); break;                                             \
        case 5: F(5); break;                                             \
        case 6: F(6); break;                                             \
        case 7: F(7); break;                                             \
        case 8: F(8); break;                                             \
        case 9: F(9); break;                                             \
        case 10: F(10); break;                                           \
        case 11: F(11); break;                                           \
        case 12: F(12); break;                                           \
        default: throw Error(-1, "unsupported order (k must be 4..12)"); \
    }

// launches of the tensor-core x step engine (instantiated only for the orders it serves)
template <int K>
static void* launch_simage(Ctx* ctx, long long nimg, const ImgSrc* d_srcs, int nt, const double* d_gblk,
                           long long nreal, cudaStream_t s) {
    if constexpr (HCfg<K>::FITS) {
        void* img = dalloc(ctx, (size_t)nimg * HCfg<K>::IMGB);
        const long long rows = nimg * (long long)HCfg<K>::R;  // one thread per data row
        k_simage<K><<<(unsigned)((rows + 255) / 256), 256, 0, s>>>(d_srcs, nt, d_gblk, nreal, nimg, (unsigned char*)img);
        return img;
    } else {
        throw Error(-1, "BF16x3 engine: unsupported order");
    }
}
template <int K>
static void launch_happly(int nchunks, const Chunk* d_chunks, const Item* d_items, const BTree* d_trees,
                          const unsigned long long* d_tkey, const unsigned long long* d_tval, const int* d_csrc,
                          const unsigned char* d_img, long long nreal, double* d_partials,
                          unsigned long long* d_ntrip, int* d_kerr, cudaStream_t s) {
    if constexpr (HCfg<K>::FITS) {
        const size_t smem = HCfg<K>::SMEM;
        MWB_CUDA(cudaFuncSetAttribute(k_happly<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_happly<K><<<nchunks, HCfg<K>::NTHR, smem, s>>>(d_chunks, d_items, d_trees, d_tkey, d_tval, d_csrc, d_img,
                                                          nreal, d_partials, d_ntrip, d_kerr);
    } else {
        throw Error(-1, "BF16x3 engine: unsupported order");
    }
}

void run_batch_pass(BatchPass& bp, cudaStream_t s) {
    const int nt = (int)bp.trees.size();
    Ctx* ctx = bp.trees[0].out->mra->ctx;
    const Mra& m = *bp.trees[0].out->mra;
    const int K = m.k;
    const size_t BS = m.bsize();
    // items (output nodes of this depth, grouped by tree) and tree descriptors
    std::vector<Item> items;
    std::vector<int> item_off(nt + 1, 0);
    std::vector<BTree> bt(nt);
    long long nreal = 0;  // block images of the input nodes at the entries' depths
    for (int t = 0; t < nt; ++t) {
        BatchTree& b = bp.trees[t];
        item_off[t] = (int)items.size();
        for (int i = b.obegin; i < b.oend; ++i) items.push_back(Item{t, i});
        Tree& o = *b.out;
        Tree& in = *b.inp;
        BTree& d = bt[t];
        d.okey = o.key;
        d.ocoef = o.coef;
        d.onorm2 = o.norm2;
        d.ownorm2 = o.wnorm2;
        d.in = InView{in.hkey, in.hval, in.hcap, in.coef, in.norm2};
        d.inkey = in.key;
        d.deltas = b.tab->d_deltas;
        d.terms = b.tab->d_terms;
        d.mats = b.tab->d_mats;
        d.mats32 = b.tab->d_mats32;
        d.matsb = b.tab->d_matsb;
        d.matsb32 = b.tab->d_matsb32;
        d.matsT = b.tab->d_matsT;
        d.matsT32 = b.tab->d_matsT32;
        d.matsbT = b.tab->d_matsbT;
        d.matsbT32 = b.tab->d_matsbT32;
        d.matsI = b.tab->d_matsI;
        d.matsbI = b.tab->d_matsbI;
        d.matsS32 = b.tab->d_matsS32;
        d.matsbS32 = b.tab->d_matsbS32;
        d.matsX = b.tab->d_matsX;
        d.nprefix = b.nprefix;
        d.root = b.depth == 0;
        d.theta = b.theta;
        // split threshold: deeper entries from the root pass's norm; root entries get theirs on the device
        d.thr = b.depth == 0 ? 0.0
                             : ((b.prec > 0.0 && b.g0 > 0.0) ? b.prec * b.g0 * std::pow(2.0, -0.5 * b.depth) : INFINITY);
        d.depth = b.depth;
        d.depth_limit = m.depth_limit;
        for (int q = 0; q < 3; ++q) d.ext[q] = (long long)m.boxes[q] << b.depth;
        d.img_lb = d.img_le = 0;
        if (in.levels() > b.depth) {
            d.img_lb = in.level_begin[b.depth];
            d.img_le = in.level_begin[b.depth + 1];
        }
        d.img_base = nreal;
        nreal += d.img_le - d.img_lb;
    }
    item_off[nt] = (int)items.size();
    const int ni = (int)items.size();
    bp.nitems = ni;
    if (ni == 0) return;
    Item* d_items = upload(ctx, items);
    BTree* d_trees = upload(ctx, bt);
    int* d_item_off = upload(ctx, item_off);

    // 1. candidates
    int* d_count = (int*)dalloc(ctx, sizeof(int) * (ni + 1));
    int* d_offs = (int*)dalloc(ctx, sizeof(int) * (ni + 1));
    int* d_ngreq = (int*)dalloc(ctx, sizeof(int));
    MWB_CUDA(cudaMemsetAsync(d_count, 0, sizeof(int) * (ni + 1), s));
    MWB_CUDA(cudaMemsetAsync(d_ngreq, 0, sizeof(int), s));
    const int cblocks = (ni * 32 + 255) / 256;
    k_bcand<<<cblocks, 256, 0, s>>>(d_items, ni, d_trees, 0, d_count, nullptr, nullptr, nullptr, nullptr, nullptr,
                                    d_ngreq);
    MWB_CUDA(cudaGetLastError());
    count(ctx);
    scan_only(ctx, d_count, d_offs, ni);
    int tot0[2] = {0, 0};  // candidates, generated-node requests: one read-back
    readback(ctx, {{&tot0[0], d_offs + ni, sizeof(int)}, {&tot0[1], d_ngreq, sizeof(int)}});
    const int ncand = tot0[0];
    const int ngreq = tot0[1];
    MWB_CUDA(cudaMemsetAsync(d_ngreq, 0, sizeof(int), s));  // the fill pass numbers the requests again
    const int ncap = std::max(1, ncand);
    int* d_cdelta = (int*)dalloc(ctx, sizeof(int) * ncap);
    int* d_csrc = (int*)dalloc(ctx, sizeof(int) * ncap);
    uint64_t* d_greq_key = (uint64_t*)dalloc(ctx, sizeof(uint64_t) * ncap);
    int* d_greq_leaf = (int*)dalloc(ctx, sizeof(int) * ncap);
    if (ncand > 0) {
        k_bcand<<<cblocks, 256, 0, s>>>(d_items, ni, d_trees, 1, d_count, d_offs, d_cdelta, d_csrc, d_greq_key,
                                        d_greq_leaf, d_ngreq);
        MWB_CUDA(cudaGetLastError());
        count(ctx);
    }

    // 2. generated nodes
    int nu = 0;
    uint64_t* d_ukey = nullptr;
    int* d_uleaf = nullptr;
    double* d_gblk = nullptr;
    double* d_gnorm2 = nullptr;
    if (ngreq > 0) {
        uint64_t* d_sk = (uint64_t*)dalloc(ctx, sizeof(uint64_t) * ngreq);
        int* d_sl = (int*)dalloc(ctx, sizeof(int) * ngreq);
        size_t tmp = 0;
        MWB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, d_greq_key, d_sk, d_greq_leaf, d_sl, ngreq, 0, 64, s));
        void* d_tmp = dalloc(ctx, tmp);
        MWB_CUDA(cub::DeviceRadixSort::SortPairs(d_tmp, tmp, d_greq_key, d_sk, d_greq_leaf, d_sl, ngreq, 0, 64, s));
        dfree(ctx, d_tmp);
        int* d_flags = (int*)dalloc(ctx, sizeof(int) * (ngreq + 1));
        int* d_pos = (int*)dalloc(ctx, sizeof(int) * (ngreq + 1));
        MWB_CUDA(cudaMemsetAsync(d_flags, 0, sizeof(int) * (ngreq + 1), s));
        k_bunique_flags<<<(ngreq + 255) / 256, 256, 0, s>>>(d_sk, ngreq, d_flags);
        nu = scan_total(ctx, d_flags, d_pos, ngreq);
        d_ukey = (uint64_t*)dalloc(ctx, sizeof(uint64_t) * nu);
        d_uleaf = (int*)dalloc(ctx, sizeof(int) * nu);
        k_bunique_scatter<<<(ngreq + 255) / 256, 256, 0, s>>>(d_sk, d_sl, d_flags, d_pos, ngreq, d_ukey, d_uleaf);
        k_bresolve_gen<<<(ncand + 255) / 256, 256, 0, s>>>(d_csrc, ncand, d_greq_key, d_ukey, nu);
        MWB_CUDA(cudaGetLastError());
        d_gblk = (double*)dalloc(ctx, sizeof(double) * (size_t)nu * K * K * K);
        d_gnorm2 = (double*)dalloc(ctx, sizeof(double) * nu);
#define L_GEN(KK)                                                                                         \
    {                                                                                                     \
        size_t smem = sizeof(double) * (Geo<KK>::VOL + 4 * KK * KK + KK * KK * KK + 64);                 \
        MWB_CUDA(cudaFuncSetAttribute(k_bgenerate<KK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
        k_bgenerate<KK><<<nu, 256, smem, s>>>(d_ukey, d_uleaf, d_trees, m.d_FT, d_gblk, d_gnorm2);            \
    }
        MWB_DISPATCH_K(K, L_GEN)
#undef L_GEN
        MWB_CUDA(cudaGetLastError());
        count(ctx, 4);
        dfree(ctx, d_sk);
        dfree(ctx, d_sl);
        dfree(ctx, d_flags);
        dfree(ctx, d_pos);
    }

    // 3-4. triples per candidate, chunks
    const bool pencil = contraction_pencil();
    // the split-TF32 engine's error floor (about 2e-7 relative, data in two TF32 pieces) stays below the
    // requested precision only from prec = 1e-6 up: finer requests take the FP32 engine
    bool tc_prec_ok = true;
    for (const BatchTree& b : bp.trees) tc_prec_ok &= !(b.prec > 0.0 && b.prec < kTensorCoreMinPrec);
    // the GEMM-tiled engine runs the line-ordered contraction (chunks of sorted triples); the
    // tensor-core and pencil engines take chunks of whole candidates
    bool lined = false, lined32 = false, hyb = false;
#define L_ENG(KK)                                                                                    \
    hyb = !pencil && bp.precision == 3 && HCfg<KK>::FITS;                                            \
    lined = hyb || (!pencil && !(bp.precision == 2 && TCfg<KK>::FITS && tc_prec_ok) &&               \
            ((bp.precision >= 1 && GCfg<KK, float>::FITS) || (bp.precision != 1 && GCfg<KK, double>::FITS))); \
    lined32 = lined && !hyb && bp.precision >= 1 && GCfg<KK, float>::FITS;
    MWB_DISPATCH_K(K, L_ENG)
#undef L_ENG
    int* d_cand_item = (int*)dalloc(ctx, sizeof(int) * ncap);
    int* d_ntrip = (int*)dalloc(ctx, sizeof(int) * (ncap + 1));
    MWB_CUDA(cudaMemsetAsync(d_ntrip, 0, sizeof(int) * (ncap + 1), s));
    if (ncand > 0) {
        k_cand_item<<<ni, 128, 0, s>>>(d_offs, ni, d_cand_item);
        k_bterms<<<(ncand + 255) / 256, 256, 0, s>>>(d_cand_item, ncand, d_items, d_trees, d_cdelta, d_csrc, d_gnorm2,
                                                     d_ntrip);
        MWB_CUDA(cudaGetLastError());
        count(ctx, 2);
    }
    int* d_nchunk = (int*)dalloc(ctx, sizeof(int) * (ni + 1));
    int* d_choff = (int*)dalloc(ctx, sizeof(int) * (ni + 1));
    int* d_nslot = (int*)dalloc(ctx, sizeof(int) * (ni + 1));
    int* d_slotoff = (int*)dalloc(ctx, sizeof(int) * (ni + 1));
    MWB_CUDA(cudaMemsetAsync(d_nchunk, 0, sizeof(int) * (ni + 1), s));
    MWB_CUDA(cudaMemsetAsync(d_nslot, 0, sizeof(int) * (ni + 1), s));
    const int chunk_limit = ctx->chunk_triples[std::min(std::max(bp.precision, 0), 3)];
    int* d_toff = nullptr;
    int* d_terr = nullptr;
    unsigned long long *d_tkey = nullptr, *d_tval = nullptr;
    void* d_ximg = nullptr;
    int nchunks = 0, nslots = 0;
    Chunk* d_chunks = nullptr;
    if (lined) {
        d_terr = (int*)dalloc(ctx, sizeof(int));
        MWB_CUDA(cudaMemsetAsync(d_terr, 0, sizeof(int), s));
        d_toff = (int*)dalloc(ctx, sizeof(int) * (ncap + 1));
        const int ntri = scan_total(ctx, d_ntrip, d_toff, ncand);
        const size_t tcap = (size_t)std::max(1, ntri);
        unsigned long long* d_tkey_in = (unsigned long long*)dalloc(ctx, sizeof(unsigned long long) * tcap);
        unsigned long long* d_tval_in = (unsigned long long*)dalloc(ctx, sizeof(unsigned long long) * tcap);
        d_tkey = (unsigned long long*)dalloc(ctx, sizeof(unsigned long long) * tcap);
        d_tval = (unsigned long long*)dalloc(ctx, sizeof(unsigned long long) * tcap);
        if (ntri > 0) {
            k_texpand<<<(ncand + 255) / 256, 256, 0, s>>>(d_offs, d_cand_item, ncand, d_items, d_trees, d_cdelta, d_ntrip,
                                                          d_toff, d_csrc, d_tkey_in, d_tval_in, d_terr);
            MWB_CUDA(cudaGetLastError());
            int hb = 1;
            while (hb < 31 && (1ll << hb) < (long long)ni) ++hb;
            size_t tmp = 0;
            MWB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, d_tkey_in, d_tkey, d_tval_in, d_tval, ntri, 0, 32 + hb, s));
            void* d_tmp = dalloc(ctx, tmp);
            MWB_CUDA(cub::DeviceRadixSort::SortPairs(d_tmp, tmp, d_tkey_in, d_tkey, d_tval_in, d_tval, ntri, 0, 32 + hb, s));
            dfree(ctx, d_tmp);
            count(ctx, 2);
        }
        dfree(ctx, d_tkey_in);
        dfree(ctx, d_tval_in);
        k_tchunks<<<(ni * 32 + 127) / 128, 128, 0, s>>>(d_offs, d_toff, ni, d_tkey, chunk_limit, 0, d_nchunk, nullptr,
                                                   nullptr, nullptr);
        k_multi_slots<<<(ni + 127) / 128, 128, 0, s>>>(d_nchunk, ni, d_nslot);
        count(ctx, 2);
        scan_only(ctx, d_nchunk, d_choff, ni);
        scan_only(ctx, d_nslot, d_slotoff, ni);
        int tot[3] = {0, 0, 0};  // chunks, partial slots, the expansion's error word: one read-back
        readback(ctx, {{&tot[0], d_choff + ni, sizeof(int)}, {&tot[1], d_slotoff + ni, sizeof(int)},
                       {&tot[2], d_terr, sizeof(int)}});
        if (tot[2] != 0) throw Error(-3, "input tree nodes are not in level order");
        nchunks = tot[0];
        nslots = tot[1];
        d_chunks = (Chunk*)dalloc(ctx, sizeof(Chunk) * std::max(1, nchunks));
        k_tchunks<<<(ni * 32 + 127) / 128, 128, 0, s>>>(d_offs, d_toff, ni, d_tkey, chunk_limit, 1, d_nchunk, d_choff,
                                                   d_slotoff, d_chunks);
        // block images of this pass's input nodes (the entries' depth levels) and generated nodes
        const long long nimg = nreal + nu;
        if (nimg > 0) {
            std::vector<ImgSrc> srcs(nt);
            for (int t = 0; t < nt; ++t)
                srcs[t] = ImgSrc{bp.trees[t].inp->coef, bt[t].img_base, bt[t].img_lb, bt[t].img_le - bt[t].img_lb};
            ImgSrc* d_srcs = upload(ctx, srcs);
#define L_IMG(KK)                                                                                               \
    {                                                                                                           \
        if (hyb) {                                                                                              \
            d_ximg = launch_simage<KK>(ctx, nimg, d_srcs, nt, d_gblk, nreal, s);                                \
        } else if (lined32) {                                                                                   \
            d_ximg = dalloc(ctx, sizeof(float) * (size_t)nimg * GCfg<KK, float>::IMG);                          \
            const int smem = (int)(sizeof(float) * 8 * KK * KK * KK);                                          \
            MWB_CUDA(cudaFuncSetAttribute(k_ximage<KK, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)); \
            k_ximage<KK, float><<<(unsigned)nimg, 256, smem, s>>>(d_srcs, nt, d_gblk, nreal, (float*)d_ximg);    \
        } else {                                                                                                \
            d_ximg = dalloc(ctx, sizeof(double) * (size_t)nimg * GCfg<KK, double>::IMG);                        \
            const int smem = (int)(sizeof(double) * 8 * KK * KK * KK);                                         \
            MWB_CUDA(cudaFuncSetAttribute(k_ximage<KK, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)); \
            k_ximage<KK, double><<<(unsigned)nimg, 256, smem, s>>>(d_srcs, nt, d_gblk, nreal, (double*)d_ximg);  \
        }                                                                                                       \
    }
            MWB_DISPATCH_K(K, L_IMG)
#undef L_IMG
            MWB_CUDA(cudaGetLastError());
            count(ctx);
            dfree(ctx, d_srcs);
        }
    } else {
        k_bchunks<<<(ni + 127) / 128, 128, 0, s>>>(d_offs, ni, d_ntrip, chunk_limit, 0, d_nchunk, nullptr, nullptr,
                                                   nullptr);
        k_multi_slots<<<(ni + 127) / 128, 128, 0, s>>>(d_nchunk, ni, d_nslot);
        count(ctx, 2);
        scan_only(ctx, d_nchunk, d_choff, ni);
        scan_only(ctx, d_nslot, d_slotoff, ni);
        int tot[2] = {0, 0};
        readback(ctx, {{&tot[0], d_choff + ni, sizeof(int)}, {&tot[1], d_slotoff + ni, sizeof(int)}});
        nchunks = tot[0];
        nslots = tot[1];
        d_chunks = (Chunk*)dalloc(ctx, sizeof(Chunk) * std::max(1, nchunks));
        k_bchunks<<<(ni + 127) / 128, 128, 0, s>>>(d_offs, ni, d_ntrip, chunk_limit, 1, d_nchunk, d_choff, d_slotoff,
                                                   d_chunks);
    }
    MWB_CUDA(cudaGetLastError());
    count(ctx);
    double* d_partials = (double*)dalloc(ctx, sizeof(double) * BS * std::max(1, nslots));
    // the line-ordered engines (tensor-core and CUDA-core) run a copy of the chunk list sorted longest
    // first, so that a launch's last wave of CTAs holds the short chunks (the reduction keeps reading the
    // list in item order)
    Chunk* d_run = d_chunks;
    if (lined && nchunks > 1) {
        int* d_len = (int*)dalloc(ctx, sizeof(int) * 2 * (size_t)nchunks);
        d_run = (Chunk*)dalloc(ctx, sizeof(Chunk) * (size_t)nchunks);
        k_chunk_len<<<(nchunks + 255) / 256, 256, 0, s>>>(d_chunks, nchunks, d_len);
        size_t tmp = 0;
        MWB_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp, d_len, d_len + nchunks, d_chunks, d_run, nchunks,
                                                           0, 16, s));
        void* d_tmp = dalloc(ctx, tmp);
        MWB_CUDA(cub::DeviceRadixSort::SortPairsDescending(d_tmp, tmp, d_len, d_len + nchunks, d_chunks, d_run, nchunks,
                                                           0, 16, s));
        dfree(ctx, d_tmp);
        dfree(ctx, d_len);
        count(ctx, 2);
    }

    // 5. contraction + reduction of multi-chunk nodes
    unsigned long long* d_ntrip_tot = (unsigned long long*)dalloc(ctx, 2 * sizeof(unsigned long long));
    int* d_kerr = reinterpret_cast<int*>(d_ntrip_tot + 1);  // set by the tensor-core kernel on a wait timeout
    MWB_CUDA(cudaMemsetAsync(d_ntrip_tot, 0, 2 * sizeof(unsigned long long), s));
    if (ctx->prof) MWB_CUDA(cudaEventRecord(ctx->ev0, s));
#define L_AP(KK)                                                                                             \
    {                                                                                                        \
        if (hyb) {                                                                                           \
            launch_happly<KK>(nchunks, d_run, d_items, d_trees, d_tkey, d_tval, d_csrc,                      \
                              (const unsigned char*)d_ximg, nreal, d_partials, d_ntrip_tot, d_kerr, s);       \
        } else if (bp.precision == 2 && TCfg<KK>::FITS && !pencil && tc_prec_ok) {                           \
            size_t smem = TCfg<KK>::SMEM;                                                                    \
            MWB_CUDA(cudaFuncSetAttribute(k_tapply<KK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
            k_tapply<KK><<<nchunks, TCfg<KK>::NTHR, smem, s>>>(d_chunks, d_items, d_trees, d_cdelta, d_csrc,     \
                                                               d_gblk, d_gnorm2, d_partials, d_ntrip_tot, d_kerr); \
        } else if (bp.precision >= 1 && GCfg<KK, float>::FITS && !pencil) {                                  \
            size_t smem = GCfg<KK, float>::SMEM;                                                             \
            MWB_CUDA(cudaFuncSetAttribute(k_gapply<KK, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
            k_gapply<KK, float><<<nchunks, GCfg<KK, float>::NTHR, smem, s>>>(d_run, d_items, d_trees, d_tkey,    \
                                                                              d_tval, d_csrc, (const float*)d_ximg, \
                                                                              nreal, d_partials, d_ntrip_tot);     \
        } else if (bp.precision != 1 && GCfg<KK, double>::FITS && !pencil) {                                  \
            size_t smem = GCfg<KK, double>::SMEM;                                                            \
            MWB_CUDA(cudaFuncSetAttribute(k_gapply<KK, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
            k_gapply<KK, double><<<nchunks, GCfg<KK, double>::NTHR, smem, s>>>(d_run, d_items, d_trees, d_tkey,   \
                                                                                d_tval, d_csrc, (const double*)d_ximg, \
                                                                                nreal, d_partials, d_ntrip_tot);    \
        } else if (bp.precision >= 1) {                                                                      \
            size_t smem = ACfg<KK, float>::SMEM;                                                             \
            MWB_CUDA(cudaFuncSetAttribute(k_bapply<KK, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
            k_bapply<KK, float><<<nchunks, ACfg<KK, float>::NT, smem, s>>>(d_chunks, d_items, d_trees, d_cdelta,  \
                                                                            d_csrc, d_gblk, d_gnorm2, d_partials, \
                                                                            d_ntrip_tot);                         \
        } else {                                                                                             \
            size_t smem = ACfg<KK, double>::SMEM;                                                            \
            MWB_CUDA(cudaFuncSetAttribute(k_bapply<KK, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
            k_bapply<KK, double><<<nchunks, ACfg<KK, double>::NT, smem, s>>>(d_chunks, d_items, d_trees, d_cdelta, \
                                                                              d_csrc, d_gblk, d_gnorm2, d_partials, \
                                                                              d_ntrip_tot);                        \
        }                                                                                                    \
    }
    MWB_DISPATCH_K(K, L_AP)
#undef L_AP
    MWB_CUDA(cudaGetLastError());
    if (ctx->prof) MWB_CUDA(cudaEventRecord(ctx->ev1, s));
    if (d_run != d_chunks) dfree(ctx, d_run);
    count(ctx);
    ctx->apply_launches++;
    ctx->apply_ctas += nchunks;
    if (nslots > 0) {  // one block per item; items whose node took one chunk leave at once
#define L_RED(KK) k_breduce<KK><<<ni, 256, 0, s>>>(d_chunks, d_choff, nullptr, d_items, d_trees, d_partials);
        MWB_DISPATCH_K(K, L_RED)
#undef L_RED
        MWB_CUDA(cudaGetLastError());
        count(ctx);
    }

    // 6. root norms and thresholds (root entries), split flags; one read-back for the pass's results
    bool any_root = false;
    for (int t = 0; t < nt; ++t) any_root |= bp.trees[t].depth == 0;
    double* d_g = nullptr;
    if (any_root) {
        d_g = (double*)dalloc(ctx, sizeof(double) * nt);
        std::vector<double> precs(nt);
        for (int t = 0; t < nt; ++t) precs[t] = bp.trees[t].prec;
        double* d_prec = upload(ctx, precs);
        k_tree_item_norm2<<<nt, 256, 0, s>>>(d_items, d_item_off, d_trees, d_g);
        k_root_thr<<<(nt + 127) / 128, 128, 0, s>>>(d_trees, d_g, d_prec, nt);
        MWB_CUDA(cudaGetLastError());
        count(ctx, 2);
        dfree(ctx, d_prec);
    }
    int* d_sflags = (int*)dalloc(ctx, sizeof(int) * (ni + 1));
    k_bsplit_flags<<<(ni + 255) / 256, 256, 0, s>>>(d_items, ni, d_trees, d_sflags);
    MWB_CUDA(cudaGetLastError());
    count(ctx);
    unsigned long long ntot[2] = {0, 0};
    std::vector<int> sflags(ni);
    std::vector<double> g(any_root ? nt : 0);
    readback(ctx, {{ntot, d_ntrip_tot, sizeof(ntot)}, {sflags.data(), d_sflags, sizeof(int) * ni},
                   {g.data(), d_g, any_root ? sizeof(double) * nt : 0}});
    if ((ntot[1] & 0xffffffffull) != 0)
        throw Error(-2, "tensor-core contraction: an MMA or copy completion wait exceeded its time limit");
    if (ctx->prof) {
        float ms = 0.0f;
        MWB_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        ctx->apply_ms += ms;
    }
    bp.triples = (long long)ntot[0];
    for (int t = 0; t < nt; ++t)
        if (bp.trees[t].depth == 0) bp.trees[t].g0 = std::sqrt(g[t]);
    bp.split_lists.assign(nt, {});
    for (int t = 0; t < nt; ++t)
        for (int i = item_off[t]; i < item_off[t + 1]; ++i)
            if (sflags[i]) bp.split_lists[t].push_back(items[i].node);
    dfree(ctx, d_g);
    for (void* p : std::initializer_list<void*>{d_items, d_trees, d_item_off, d_count, d_offs, d_ngreq, d_cdelta, d_csrc,
                                                d_greq_key, d_greq_leaf, d_ukey, d_uleaf, d_gblk, d_gnorm2, d_cand_item,
                                                d_ntrip, d_nchunk, d_choff, d_nslot, d_slotoff, d_chunks, d_partials,
                                                d_ntrip_tot, d_sflags, d_toff, d_tkey, d_tval, d_terr, d_ximg})
        dfree(ctx, p);
    bp.nchunks = nchunks;
    bp.nslots = nslots;
}

}  // namespace mwb
