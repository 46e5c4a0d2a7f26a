// mw_apply.cu -- batched, adaptive NS-form apply on the device.
//
// A batch is any number of (output tree, operator, input tree) triples sharing one world (e.g. 32
// orbitals with 32 Helmholtz operators).  The refinement passes run in lock-step over the batch:
// pass d handles the depth-d output nodes of every tree with one launch per stage:
//   1. candidates: one warp per output node walks its operator's offset list, looks the input node
//      up in the input tree's hash index (or its leaf ancestor -> generated node) and screens it;
//   2. generated (scaling-only) input nodes are de-duplicated per tree and built once;
//   3. per candidate, the number of terms that pass the screening (the triples it contributes);
//   4. each output node's candidate list is cut into chunks of at most kChunkTriples triples;
//   5. the contraction kernel runs one CTA per chunk; multi-chunk nodes write partial blocks that
//      a reduction kernel adds in chunk order (deterministic), single-chunk nodes write directly;
//   6. norms and split flags; children are appended to each tree.
// Results are identical to the per-node sequential order up to FP64 rounding.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>

#include "mw_device.cuh"
#include "mw_kernels.cuh"

namespace mwb {

constexpr int kChunkTriples = 48;  // triples per contraction CTA (load balance vs partial traffic)

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
    int nprefix;
    int root;
    double theta;
    double thr;  // split threshold of this pass
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
__global__ void k_bcand(const Item* __restrict__ items, int nitems, const BTree* __restrict__ trees, int depth,
                        long long e0, long long e1, long long e2, int fill, int* count, const int* offs, int* cdelta,
                        int* csrc, uint64_t* greq_key, int* greq_leaf, int* ngreq) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x & 31;
    if (w >= nitems) return;
    const Item it = items[w];
    const BTree& T = trees[it.tree];
    const long long ext[3] = {e0, e1, e2};
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
                        // tree index in the (per-pass constant) depth bits: unique across the batch
                        gk = ((uint64_t)it.tree << 57) | (key & ((1ull << 57) - 1));
                    }
                }
            }
        }
        const unsigned bal = __ballot_sync(0xffffffffu, ok);
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
template <int K>
__global__ void __launch_bounds__(256) k_bgenerate(const uint64_t* __restrict__ ukey, const int* __restrict__ uleaf,
                                                   const BTree* __restrict__ trees, int depth,
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
    const int leaf = uleaf[g];
    for (int i = threadIdx.x; i < G::K2 * G::K2; i += blockDim.x) M[i] = FT[i];
    for (int e = threadIdx.x; e < G::BS; e += blockDim.x) {
        const int a = e % G::K2, b = (e / G::K2) % G::K2, c = e / (G::K2 * G::K2);
        A[G::at(a, b, c)] = T.in.coef[(size_t)leaf * G::BS + e];
    }
    __syncthreads();
    pencil_transform<K, 0>(M, A);
    __syncthreads();
    pencil_transform<K, 1>(M, A);
    __syncthreads();
    pencil_transform<K, 2>(M, A);
    __syncthreads();
    long long t[3], tl[3];
    key_trans(gkey & ((1ull << 57) - 1), t);
    key_trans(T.inkey[leaf], tl);
    const int dl = depth - key_depth(T.inkey[leaf]);
    int cc[3];
    for (int q = 0; q < 3; ++q) cc[q] = (int)((t[q] >> (dl - 1)) - 2 * tl[q]);
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
// greedy cut of each node's candidates into chunks of at most kChunkTriples triples (whole
// candidates; at least one chunk per node so that every output block gets written)
__global__ void k_bchunks(const int* __restrict__ offs, int nitems, const int* __restrict__ ntrip, int fill,
                          int* nchunk, const int* __restrict__ choff, const int* __restrict__ slotoff, Chunk* chunks) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nitems) return;
    const int c0 = offs[w], c1 = offs[w + 1];
    int nch = 0, acc = 0, start = c0;
    const int multi = fill ? (choff[w + 1] - choff[w] > 1) : 0;
    for (int c = c0; c < c1; ++c) {
        const int t = ntrip[c];
        if (acc > 0 && acc + t > kChunkTriples) {
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

// ---------------------------------------------------------------------------------------------
// 5. FP64 contraction (one CTA per chunk)
// ---------------------------------------------------------------------------------------------
template <int K>
struct ApplyCfg {
    static constexpr int K2 = 2 * K;
    static constexpr int NP = K2 * K2;
    static constexpr bool STAGE = K2 <= 20;       // input block staged in shared memory
    static constexpr int PPT = K2 <= 20 ? 1 : 2;   // z-pencils (accumulators) per thread
    static constexpr int NT = ((NP + PPT - 1) / PPT + 31) / 32 * 32;
    static constexpr int XS = STAGE ? Geo<K>::VOL : K * K * K;
    static constexpr size_t SMEM = sizeof(double) * (size_t)(XS + Geo<K>::VOL + 3 * NP + K * K * K + 64);
};

template <int K, bool GEN>
__device__ __forceinline__ double xin(const double* X, const double* __restrict__ blk, int a, int b, int c) {
    using C = ApplyCfg<K>;
    if (C::STAGE) return X[Geo<K>::at(a, b, c)];
    if (GEN) return X[a + K * (b + K * c)];
    return __ldg(&blk[a + 2 * K * (b + 2 * K * c)]);
}

// x-step: T[:, b, c] = M_x X[:, b, c] (GEN: k scaling inputs, b, c < k), and for depth > 0 the
// scaling-only chain U = T_x X_sss
template <int K, bool GEN>
__device__ __forceinline__ void step_x(const double* __restrict__ Mx, const double* X, const double* __restrict__ blk,
                                       double* T, double* U, bool root) {
    using G = Geo<K>;
    constexpr int K2 = G::K2;
    constexpr int NIN = GEN ? K : K2;
    constexpr int UX = GEN ? K : K2;
    for (int p = threadIdx.x; p < UX * UX; p += blockDim.x) {
        const int b = p % UX, c = p / UX;
        double x[NIN];
#pragma unroll
        for (int i = 0; i < NIN; ++i) x[i] = xin<K, GEN>(X, blk, i, b, c);
#pragma unroll 2
        for (int o = 0; o < K2; ++o) {
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < NIN; ++i) s = fma(Mx[o * K2 + i], x[i], s);
            T[G::at(o, b, c)] = s;
        }
    }
    if (!root) {
        for (int p = threadIdx.x; p < K * K; p += blockDim.x) {
            const int b = p % K, c = p / K;
            double x[K];
#pragma unroll
            for (int i = 0; i < K; ++i) x[i] = xin<K, GEN>(X, blk, i, b, c);
#pragma unroll 2
            for (int o = 0; o < K; ++o) {
                double s = 0.0;
#pragma unroll
                for (int i = 0; i < K; ++i) s = fma(Mx[o * K2 + i], x[i], s);
                U[o + K * (b + K * c)] = s;
            }
        }
    }
}

template <int K, bool GEN>
__device__ __forceinline__ void step_y(const double* __restrict__ My, double* T, double* U, bool root) {
    using G = Geo<K>;
    constexpr int K2 = G::K2;
    constexpr int NIN = GEN ? K : K2;
    constexpr int NC = GEN ? K : K2;
    for (int p = threadIdx.x; p < K2 * NC; p += blockDim.x) {
        const int a = p % K2, c = p / K2;
        double x[NIN];
#pragma unroll
        for (int i = 0; i < NIN; ++i) x[i] = T[G::at(a, i, c)];
#pragma unroll 2
        for (int o = 0; o < K2; ++o) {
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < NIN; ++i) s = fma(My[o * K2 + i], x[i], s);
            T[G::at(a, o, c)] = s;
        }
    }
    if (!root) {
        for (int p = threadIdx.x; p < K * K; p += blockDim.x) {
            const int a = p % K, c = p / K;
            double x[K];
#pragma unroll
            for (int i = 0; i < K; ++i) x[i] = U[a + K * (i + K * c)];
#pragma unroll 2
            for (int o = 0; o < K; ++o) {
                double s = 0.0;
#pragma unroll
                for (int i = 0; i < K; ++i) s = fma(My[o * K2 + i], x[i], s);
                U[a + K * (o + K * c)] = s;
            }
        }
    }
}

template <int K, bool GEN>
__device__ __forceinline__ void step_z(const double* __restrict__ Mz, const double* T, const double* U, bool root,
                                       double beta, double (&acc)[ApplyCfg<K>::PPT][2 * K]) {
    using G = Geo<K>;
    using C = ApplyCfg<K>;
    constexpr int K2 = G::K2;
    constexpr int NIN = GEN ? K : K2;
#pragma unroll
    for (int j = 0; j < C::PPT; ++j) {
        const int p = threadIdx.x + j * C::NT;
        if (p < C::NP) {
            const int a = p % K2, b = p / K2;
            double x[NIN];
#pragma unroll
            for (int i = 0; i < NIN; ++i) x[i] = T[G::at(a, b, i)];
#pragma unroll
            for (int o = 0; o < K2; ++o) {
                double s = 0.0;
#pragma unroll
                for (int i = 0; i < NIN; ++i) s = fma(Mz[o * K2 + i], x[i], s);
                acc[j][o] = fma(beta, s, acc[j][o]);
            }
            if (!root && a < K && b < K) {
                double u[K];
#pragma unroll
                for (int i = 0; i < K; ++i) u[i] = U[a + K * (b + K * i)];
#pragma unroll
                for (int o = 0; o < K; ++o) {
                    double s = 0.0;
#pragma unroll
                    for (int i = 0; i < K; ++i) s = fma(Mz[o * K2 + i], u[i], s);
                    acc[j][o] = fma(-beta, s, acc[j][o]);
                }
            }
        }
    }
}

// For every term of every candidate of the chunk:
//   out += beta (NS_z (x) NS_y (x) NS_x) in        (three in-place pencil transforms)
//   out_sss -= beta (T_z (x) T_y (x) T_x) in_sss   (depth > 0: the s->s block belongs to coarser scales)
template <int K>
__global__ void __launch_bounds__(ApplyCfg<K>::NT, 1)
    k_bapply_fp64(const Chunk* __restrict__ chunks, const Item* __restrict__ items, const BTree* __restrict__ trees,
                  const int* __restrict__ cdelta, const int* __restrict__ csrc, const double* __restrict__ gblk,
                  const double* __restrict__ gnorm2, double* partials, unsigned long long* ntrip_out) {
    using G = Geo<K>;
    using C = ApplyCfg<K>;
    constexpr int K2 = G::K2;
    extern __shared__ double sm[];
    double* X = sm;
    double* T = X + C::XS;
    double* Mx = T + G::VOL;
    double* My = Mx + C::NP;
    double* Mz = My + C::NP;
    double* U = Mz + C::NP;
    double* red = U + K * K * K;
    const Chunk ch = chunks[blockIdx.x];
    const Item it = items[ch.item];
    const BTree& TR = trees[it.tree];
    const bool root = TR.root != 0;
    const double theta = TR.theta;
    const int tid = threadIdx.x;
    double acc[C::PPT][K2];
#pragma unroll
    for (int j = 0; j < C::PPT; ++j)
#pragma unroll
        for (int c = 0; c < K2; ++c) acc[j][c] = 0.0;
    unsigned long long ntrip = 0;
    for (int ci = ch.c0; ci < ch.c1; ++ci) {
        const int src = csrc[ci];
        const bool gen = src < 0;
        const double nu = gen ? sqrt(gnorm2[-src - 1]) : sqrt(TR.in.norm2[src]);
        const DeltaRec de = TR.deltas[cdelta[ci]];
        if (!(nu > 0.0) || de.maxb * nu < theta) continue;
        if (TR.terms[de.t0].bound * nu < theta) continue;
        const double* blk = gen ? gblk + (size_t)(-src - 1) * K * K * K : TR.in.coef + (size_t)src * G::BS;
        __syncthreads();  // previous candidate's users of X/T/U/M are done
        if (gen) {
            for (int e2 = tid; e2 < K * K * K; e2 += blockDim.x) {
                const int a = e2 % K, b = (e2 / K) % K, c = e2 / (K * K);
                if (C::STAGE) X[G::at(a, b, c)] = blk[e2]; else X[e2] = blk[e2];
            }
        } else if (C::STAGE) {
            for (int e2 = tid; e2 < G::BS; e2 += blockDim.x) {
                const int a = e2 % K2, b = (e2 / K2) % K2, c = e2 / (K2 * K2);
                X[G::at(a, b, c)] = blk[e2];
            }
        }
        for (int ti = de.t0; ti < de.t1; ++ti) {
            const TermRec tr = TR.terms[ti];
            if (tr.bound * nu < theta) break;
            __syncthreads();
            for (int i = tid; i < C::NP; i += blockDim.x) {
                Mx[i] = TR.mats[(size_t)tr.mx * C::NP + i];
                My[i] = TR.mats[(size_t)tr.my * C::NP + i];
                Mz[i] = TR.mats[(size_t)tr.mz * C::NP + i];
            }
            __syncthreads();
            if (gen) step_x<K, true>(Mx, X, blk, T, U, root); else step_x<K, false>(Mx, X, blk, T, U, root);
            __syncthreads();
            if (gen) step_y<K, true>(My, T, U, root); else step_y<K, false>(My, T, U, root);
            __syncthreads();
            if (gen) step_z<K, true>(Mz, T, U, root, tr.beta, acc); else step_z<K, false>(Mz, T, U, root, tr.beta, acc);
            ++ntrip;
        }
    }
    double* dst = ch.slot < 0 ? TR.ocoef + (size_t)it.node * G::BS : partials + (size_t)ch.slot * G::BS;
    double n2 = 0.0, w2 = 0.0;
#pragma unroll
    for (int j = 0; j < C::PPT; ++j) {
        const int p = tid + j * C::NT;
        if (p < C::NP) {
            const int a = p % K2, b = p / K2;
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

// add the partial blocks of a multi-chunk node in chunk order; write block and norms
template <int K>
__global__ void __launch_bounds__(256) k_breduce(const Chunk* __restrict__ chunks, const int* __restrict__ choff,
                                                 const int* __restrict__ multi_items, const Item* __restrict__ items,
                                                 const BTree* __restrict__ trees, const double* __restrict__ partials) {
    using G = Geo<K>;
    __shared__ double red[64];
    const int w = multi_items[blockIdx.x];
    const Item it = items[w];
    const BTree& TR = trees[it.tree];
    const int cb = choff[w], ce = choff[w + 1];
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
__global__ void k_multi_flags(const int* __restrict__ choff, int nitems, int* flags) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nitems) return;
    flags[w] = (choff[w + 1] - choff[w] > 1) ? 1 : 0;
}
__global__ void k_list_from_flags(const int* __restrict__ flags, const int* __restrict__ pos, int n, int* list) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (flags[i]) list[pos[i]] = i;
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
__global__ void k_bsplit_flags(const Item* __restrict__ items, int nitems, const BTree* __restrict__ trees, int depth,
                               int depth_limit, int* flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nitems) return;
    const Item it = items[i];
    const BTree& T = trees[it.tree];
    flags[i] = (depth < depth_limit && sqrt(T.ownorm2[it.node]) > T.thr) ? 1 : 0;
}
__global__ void k_bsplit_list(const int* __restrict__ flags, const int* __restrict__ pos, const Item* __restrict__ items,
                              int n, int* list) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (flags[i]) list[pos[i]] = items[i].node;
}
__global__ void k_gather_int(const int* __restrict__ src, const int* __restrict__ idx, int n, int* dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[idx[i]];
}

// ---------------------------------------------------------------------------------------------
// driver
// ---------------------------------------------------------------------------------------------

static inline void count(Ctx* c, int n = 1) { c->launches += n; }

template <typename T>
static T* upload(Ctx* ctx, const std::vector<T>& v) {
    T* d = (T*)dalloc(ctx, sizeof(T) * std::max<size_t>(1, v.size()));
    if (!v.empty()) MWB_CUDA(cudaMemcpyAsync(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, ctx->stream));
    return d;
}
static int scan_total(Ctx* ctx, const int* d_in, int* d_out, int n) {
    size_t tmp = 0;
    MWB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, d_in, d_out, n + 1, ctx->stream));
    void* d_tmp = dalloc(ctx, tmp);
    MWB_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp, tmp, d_in, d_out, n + 1, ctx->stream));
    dfree(ctx, d_tmp);
    int total = 0;
    MWB_CUDA(cudaMemcpyAsync(&total, d_out + n, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    MWB_CUDA(cudaStreamSynchronize(ctx->stream));
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
        d.nprefix = b.nprefix;
        d.root = bp.depth == 0;
        d.theta = b.theta;
        d.thr = 0.0;
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
    const long long e0 = (long long)m.boxes[0] << bp.depth, e1 = (long long)m.boxes[1] << bp.depth,
                    e2 = (long long)m.boxes[2] << bp.depth;
    const int cblocks = (ni * 32 + 255) / 256;
    k_bcand<<<cblocks, 256, 0, s>>>(d_items, ni, d_trees, bp.depth, e0, e1, e2, 0, d_count, nullptr, nullptr, nullptr,
                                    nullptr, nullptr, nullptr);
    MWB_CUDA(cudaGetLastError());
    count(ctx);
    const int ncand = scan_total(ctx, d_count, d_offs, ni);
    const int ncap = std::max(1, ncand);
    int* d_cdelta = (int*)dalloc(ctx, sizeof(int) * ncap);
    int* d_csrc = (int*)dalloc(ctx, sizeof(int) * ncap);
    uint64_t* d_greq_key = (uint64_t*)dalloc(ctx, sizeof(uint64_t) * ncap);
    int* d_greq_leaf = (int*)dalloc(ctx, sizeof(int) * ncap);
    if (ncand > 0) {
        k_bcand<<<cblocks, 256, 0, s>>>(d_items, ni, d_trees, bp.depth, e0, e1, e2, 1, d_count, d_offs, d_cdelta, d_csrc,
                                        d_greq_key, d_greq_leaf, d_ngreq);
        MWB_CUDA(cudaGetLastError());
        count(ctx);
    }
    int ngreq = 0;
    MWB_CUDA(cudaMemcpyAsync(&ngreq, d_ngreq, sizeof(int), cudaMemcpyDeviceToHost, s));
    MWB_CUDA(cudaStreamSynchronize(s));

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
        k_bgenerate<KK><<<nu, 256, smem, s>>>(d_ukey, d_uleaf, d_trees, bp.depth, m.d_FT, d_gblk, d_gnorm2); \
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
    int* d_cand_item = (int*)dalloc(ctx, sizeof(int) * ncap);
    int* d_ntrip = (int*)dalloc(ctx, sizeof(int) * ncap);
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
    k_bchunks<<<(ni + 127) / 128, 128, 0, s>>>(d_offs, ni, d_ntrip, 0, d_nchunk, nullptr, nullptr, nullptr);
    k_multi_slots<<<(ni + 127) / 128, 128, 0, s>>>(d_nchunk, ni, d_nslot);
    count(ctx, 2);
    const int nchunks = scan_total(ctx, d_nchunk, d_choff, ni);
    const int nslots = scan_total(ctx, d_nslot, d_slotoff, ni);
    Chunk* d_chunks = (Chunk*)dalloc(ctx, sizeof(Chunk) * std::max(1, nchunks));
    k_bchunks<<<(ni + 127) / 128, 128, 0, s>>>(d_offs, ni, d_ntrip, 1, d_nchunk, d_choff, d_slotoff, d_chunks);
    MWB_CUDA(cudaGetLastError());
    count(ctx);
    double* d_partials = (double*)dalloc(ctx, sizeof(double) * BS * std::max(1, nslots));

    // 5. contraction + reduction of multi-chunk nodes
    unsigned long long* d_ntrip_tot = (unsigned long long*)dalloc(ctx, sizeof(unsigned long long));
    MWB_CUDA(cudaMemsetAsync(d_ntrip_tot, 0, sizeof(unsigned long long), s));
    if (ctx->prof) MWB_CUDA(cudaEventRecord(ctx->ev0, s));
#define L_AP(KK)                                                                                            \
    {                                                                                                       \
        size_t smem = ApplyCfg<KK>::SMEM;                                                                   \
        MWB_CUDA(cudaFuncSetAttribute(k_bapply_fp64<KK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
        k_bapply_fp64<KK><<<nchunks, ApplyCfg<KK>::NT, smem, s>>>(d_chunks, d_items, d_trees, d_cdelta, d_csrc,  \
                                                                   d_gblk, d_gnorm2, d_partials, d_ntrip_tot);  \
    }
    MWB_DISPATCH_K(K, L_AP)
#undef L_AP
    MWB_CUDA(cudaGetLastError());
    if (ctx->prof) MWB_CUDA(cudaEventRecord(ctx->ev1, s));
    count(ctx);
    ctx->apply_launches++;
    if (nslots > 0) {
        int* d_mflags = (int*)dalloc(ctx, sizeof(int) * (ni + 1));
        int* d_mpos = (int*)dalloc(ctx, sizeof(int) * (ni + 1));
        MWB_CUDA(cudaMemsetAsync(d_mflags, 0, sizeof(int) * (ni + 1), s));
        k_multi_flags<<<(ni + 255) / 256, 256, 0, s>>>(d_choff, ni, d_mflags);
        const int nmulti = scan_total(ctx, d_mflags, d_mpos, ni);
        int* d_mlist = (int*)dalloc(ctx, sizeof(int) * std::max(1, nmulti));
        k_list_from_flags<<<(ni + 255) / 256, 256, 0, s>>>(d_mflags, d_mpos, ni, d_mlist);
#define L_RED(KK) k_breduce<KK><<<nmulti, 256, 0, s>>>(d_chunks, d_choff, d_mlist, d_items, d_trees, d_partials);
        MWB_DISPATCH_K(K, L_RED)
#undef L_RED
        MWB_CUDA(cudaGetLastError());
        count(ctx, 3);
        dfree(ctx, d_mflags);
        dfree(ctx, d_mpos);
        dfree(ctx, d_mlist);
    }
    unsigned long long ntot = 0;
    MWB_CUDA(cudaMemcpyAsync(&ntot, d_ntrip_tot, sizeof(ntot), cudaMemcpyDeviceToHost, s));
    MWB_CUDA(cudaStreamSynchronize(s));
    if (ctx->prof) {
        float ms = 0.0f;
        MWB_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        ctx->apply_ms += ms;
    }
    bp.triples = (long long)ntot;

    // 6. root norms (g0 per tree) when needed, then split lists per tree
    if (bp.depth == 0) {
        double* d_g = (double*)dalloc(ctx, sizeof(double) * nt);
        k_tree_item_norm2<<<nt, 256, 0, s>>>(d_items, d_item_off, d_trees, d_g);
        count(ctx);
        std::vector<double> g(nt);
        MWB_CUDA(cudaMemcpyAsync(g.data(), d_g, sizeof(double) * nt, cudaMemcpyDeviceToHost, s));
        MWB_CUDA(cudaStreamSynchronize(s));
        for (int t = 0; t < nt; ++t) bp.trees[t].g0 = std::sqrt(g[t]);
        dfree(ctx, d_g);
    }
    for (int t = 0; t < nt; ++t) {
        const BatchTree& b = bp.trees[t];
        bt[t].thr = (b.prec > 0.0 && b.g0 > 0.0) ? b.prec * b.g0 * std::pow(2.0, -0.5 * bp.depth) : INFINITY;
    }
    MWB_CUDA(cudaMemcpyAsync(d_trees, bt.data(), sizeof(BTree) * nt, cudaMemcpyHostToDevice, s));
    int* d_sflags = (int*)dalloc(ctx, sizeof(int) * (ni + 1));
    int* d_spos = (int*)dalloc(ctx, sizeof(int) * (ni + 1));
    MWB_CUDA(cudaMemsetAsync(d_sflags, 0, sizeof(int) * (ni + 1), s));
    k_bsplit_flags<<<(ni + 255) / 256, 256, 0, s>>>(d_items, ni, d_trees, bp.depth, m.depth_limit, d_sflags);
    count(ctx);
    const int nsplit = scan_total(ctx, d_sflags, d_spos, ni);
    bp.split_lists.assign(nt, {});
    if (nsplit > 0) {
        int* d_slist = (int*)dalloc(ctx, sizeof(int) * nsplit);
        k_bsplit_list<<<(ni + 255) / 256, 256, 0, s>>>(d_sflags, d_spos, d_items, ni, d_slist);
        int* d_bpos = (int*)dalloc(ctx, sizeof(int) * (nt + 1));
        k_gather_int<<<1, 256, 0, s>>>(d_spos, d_item_off, nt + 1, d_bpos);
        count(ctx, 2);
        std::vector<int> bpos(nt + 1), slist(nsplit);
        MWB_CUDA(cudaMemcpyAsync(bpos.data(), d_bpos, sizeof(int) * (nt + 1), cudaMemcpyDeviceToHost, s));
        MWB_CUDA(cudaMemcpyAsync(slist.data(), d_slist, sizeof(int) * nsplit, cudaMemcpyDeviceToHost, s));
        MWB_CUDA(cudaStreamSynchronize(s));
        for (int t = 0; t < nt; ++t) bp.split_lists[t].assign(slist.begin() + bpos[t], slist.begin() + bpos[t + 1]);
        dfree(ctx, d_slist);
        dfree(ctx, d_bpos);
    }
    for (void* p : std::initializer_list<void*>{d_items, d_trees, d_item_off, d_count, d_offs, d_ngreq, d_cdelta, d_csrc,
                                                d_greq_key, d_greq_leaf, d_ukey, d_uleaf, d_gblk, d_gnorm2, d_cand_item,
                                                d_ntrip, d_nchunk, d_choff, d_nslot, d_slotoff, d_chunks, d_partials,
                                                d_ntrip_tot, d_sflags, d_spos})
        dfree(ctx, p);
    bp.nchunks = nchunks;
    bp.nslots = nslots;
}

}  // namespace mwb
