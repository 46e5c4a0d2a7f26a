// mw_multiply.cu -- pointwise product of two functions on the device (multiwavelet multiplication)
// and the union-grid helpers it is used with.
//
// Contract: mrcpp::multiply(prec, out, c, a, b[, maxIter]) and mrcpp::build_grid / copy_grid as called
// at reference src/qmfunctions/qmfunction_utils.cpp:209-217 (union grid: build_grid(out, a),
// build_grid(out, b), multiply(..., maxIter = 0); adaptive: multiply on the output's current grid,
// refined until converged), src/qmoperators/two_electron/ExchangePotential.cpp:131,253,312 and
// src/qmfunctions/density_utils.cpp:65-91 (square).
//
// Per output node (scale n): both factors are taken at scale n+1 on the node's 8 children -- the
// reconstructed node block, or, where a factor's tree is coarser, the block generated below its
// deepest existing ancestor (zero wavelets) -- evaluated at the children's k^3 Gauss-Legendre points
// (one (2k)x(2k) matrix per dimension, MV = blkdiag(E, E) F^T), multiplied, and projected back and
// compressed with the projection matrix PF = F blkdiag(W, W) and the scale c 2^{3(n+1)/2}.
// Refinement follows the adaptive projection: after every pass the leaves whose wavelet norm exceeds
// prec ||out|| 2^{-depth/2} are split and their children computed.
//
// Work per node: 9 to 9 + 6 L in-place pencil transforms of a (2k)^3 FP64 tensor (L = levels of
// generation), 2 blocks read and 1 written: compute-bound on the FP64 pipe, off the apply's hot path.
#include <algorithm>
#include <cmath>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/mwb200.h"
#include "mw_device.cuh"
#include "mw_kernels.cuh"
#include "mw_learned.cuh"

namespace mwb {

void set_last_error(const std::string& msg);

struct MulTree {
    uint64_t* okey;
    double* ocoef;
    double* onorm2;
    double* ownorm2;
    const uint64_t* ahk;
    const int* ahv;
    uint32_t ahcap;
    const double* acoef;
    const uint64_t* bhk;
    const int* bhv;
    uint32_t bhcap;
    const double* bcoef;
    double c;
};

struct MulItem {
    int tree;
    int node;
};

constexpr int kMulThreads = 416;  // 13 warps: one pencil of a (2k)^3 block per thread at k = 10

template <int K>
struct MulCfg {
    using G = Geo<K>;
    static constexpr int K2 = 2 * K;
    static constexpr int KKK = K * K * K;
    static constexpr int PER = (KKK + kMulThreads - 1) / kMulThreads;  // octant values per thread
    static constexpr size_t SMEM = sizeof(double) * (2 * (size_t)G::VOL + 3 * K2 * K2 + 64) + 16;
    static constexpr bool FITS = SMEM <= 227 * 1024;
};

// Block of a factor at node `key` into the padded tensor T: the node's own compressed block, or the
// scaling-only block generated below the deepest existing ancestor.  `slot` is a shared int.
template <int K>
__device__ void mul_fetch(double* T, const double* FT, const uint64_t* hk, const int* hv, uint32_t hcap,
                          const double* coef, uint64_t key, int* slot) {
    using G = Geo<K>;
    using C = MulCfg<K>;
    const int depth = key_depth(key);
    long long tr[3];
    key_trans(key, tr);
    if (threadIdx.x == 0) {
        int idx = hlookup(hk, hv, hcap, key), da = depth;
        while (idx < 0 && da > 0) {
            --da;
            const int sh = depth - da;
            idx = hlookup(hk, hv, hcap, make_key(da, tr[0] >> sh, tr[1] >> sh, tr[2] >> sh));
        }
        slot[0] = idx;
        slot[1] = da;
    }
    __syncthreads();
    const int idx = slot[0], da = slot[1];
    if (idx < 0) {  // outside the factor's roots (cannot happen on one world): zero
        for (int e = threadIdx.x; e < G::VOL; e += blockDim.x) T[e] = 0.0;
        return;
    }
    const double* blk = coef + (size_t)idx * G::BS;
    for (int e = threadIdx.x; e < G::BS; e += blockDim.x) {
        const int a = e % G::K2, b = (e / G::K2) % G::K2, c = e / (G::K2 * G::K2);
        T[G::at(a, b, c)] = blk[e];
    }
    for (int lev = da; lev < depth; ++lev) {
        // reconstruct to the children's scaling parts, keep the child on the path (zero wavelets)
        __syncthreads();
        pencil_transform<K, 0>(FT, T);
        __syncthreads();
        pencil_transform<K, 1>(FT, T);
        __syncthreads();
        pencil_transform<K, 2>(FT, T);
        __syncthreads();
        const int sh = depth - lev - 1;
        const int cx = (int)((tr[0] >> sh) & 1), cy = (int)((tr[1] >> sh) & 1), cz = (int)((tr[2] >> sh) & 1);
        double v[C::PER];
#pragma unroll
        for (int r = 0; r < C::PER; ++r) {
            const int e = threadIdx.x + r * kMulThreads;
            v[r] = 0.0;
            if (e < C::KKK) {
                const int x = e % K, y = (e / K) % K, z = e / (K * K);
                v[r] = T[G::at(cx * K + x, cy * K + y, cz * K + z)];
            }
        }
        __syncthreads();
        for (int e = threadIdx.x; e < G::VOL; e += blockDim.x) T[e] = 0.0;
        __syncthreads();
#pragma unroll
        for (int r = 0; r < C::PER; ++r) {
            const int e = threadIdx.x + r * kMulThreads;
            if (e < C::KKK) {
                const int x = e % K, y = (e / K) % K, z = e / (K * K);
                T[G::at(x, y, z)] = v[r];
            }
        }
    }
}

template <int K>
__global__ void __launch_bounds__(kMulThreads) k_mul(const MulItem* __restrict__ items, const MulTree* __restrict__ trees,
                                                     const double* __restrict__ MVg, const double* __restrict__ PFg,
                                                     const double* __restrict__ FTg, int n0) {
    using G = Geo<K>;
    constexpr int K2 = G::K2;
    extern __shared__ __align__(16) double msm[];
    double* TA = msm;
    double* TB = TA + G::VOL;
    double* MV = TB + G::VOL;
    double* PF = MV + K2 * K2;
    double* FT = PF + K2 * K2;
    double* red = FT + K2 * K2;
    int* slot = reinterpret_cast<int*>(red + 64);
    const MulItem it = items[blockIdx.x];
    const MulTree& T = trees[it.tree];
    for (int i = threadIdx.x; i < K2 * K2; i += blockDim.x) {
        MV[i] = MVg[i];
        PF[i] = PFg[i];
        FT[i] = FTg[i];
    }
    const uint64_t key = T.okey[it.node];
    __syncthreads();
    mul_fetch<K>(TA, FT, T.ahk, T.ahv, T.ahcap, T.acoef, key, slot);
    __syncthreads();
    mul_fetch<K>(TB, FT, T.bhk, T.bhv, T.bhcap, T.bcoef, key, slot);
    __syncthreads();
    // values of both factors at the children's quadrature points
    pencil_transform<K, 0>(MV, TA);
    pencil_transform<K, 0>(MV, TB);
    __syncthreads();
    pencil_transform<K, 1>(MV, TA);
    pencil_transform<K, 1>(MV, TB);
    __syncthreads();
    pencil_transform<K, 2>(MV, TA);
    pencil_transform<K, 2>(MV, TB);
    __syncthreads();
    for (int e = threadIdx.x; e < G::VOL; e += blockDim.x) TA[e] *= TB[e];
    __syncthreads();
    pencil_transform<K, 0>(PF, TA);
    __syncthreads();
    pencil_transform<K, 1>(PF, TA);
    __syncthreads();
    // last dimension in registers, scaled, written with the block norms
    const double fac = T.c * exp2(1.5 * (double)(n0 + key_depth(key) + 1));
    double* dst = T.ocoef + (size_t)it.node * G::BS;
    double n2 = 0.0, w2 = 0.0;
    for (int p = threadIdx.x; p < G::NP; p += blockDim.x) {
        const int a = p % K2, b = p / K2;
        double x[K2];
#pragma unroll
        for (int i = 0; i < K2; ++i) x[i] = TA[G::at(a, b, i)];
#pragma unroll 1
        for (int o = 0; o < K2; ++o) {
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < K2; ++i) s = fma(PF[o * K2 + i], x[i], s);
            s *= fac;
            dst[a + K2 * (b + K2 * o)] = s;
            n2 += s * s;
            if (!(a < K && b < K && o < K)) w2 += s * s;
        }
    }
    block_sum2(n2, w2, red);
    if (threadIdx.x == 0) {
        T.onorm2[it.node] = n2;
        T.ownorm2[it.node] = w2;
    }
}

// linear combination: one input function of a sum
struct AddIn {
    const uint64_t* hk;
    const int* hv;
    uint32_t hcap;
    const double* coef;
    double c;
};
struct AddOut {
    const uint64_t* key;
    double* coef;
    double* norm2;
    double* wnorm2;
};
constexpr int kAddMaxTerms = 256;

// block of sum_i c_i f_i at one output node: compressed blocks are linear in the function, so the
// inputs' blocks (own, or generated below the deepest ancestor) are combined as they are
template <int K>
__global__ void __launch_bounds__(kMulThreads) k_add(const MulItem* __restrict__ items, AddOut out,
                                                     const AddIn* __restrict__ in, int nin,
                                                     const double* __restrict__ FTg) {
    using G = Geo<K>;
    constexpr int K2 = G::K2;
    extern __shared__ __align__(16) double asm_[];
    double* ACC = asm_;
    double* T = ACC + G::VOL;
    double* FT = T + G::VOL;
    double* unused = FT + K2 * K2;
    double* red = unused + K2 * K2;
    int* slot = reinterpret_cast<int*>(red + 64);
    const int node = items[blockIdx.x].node;
    for (int i = threadIdx.x; i < K2 * K2; i += blockDim.x) FT[i] = FTg[i];
    for (int e = threadIdx.x; e < G::VOL; e += blockDim.x) ACC[e] = 0.0;
    const uint64_t key = out.key[node];
    __syncthreads();
    for (int q = 0; q < nin; ++q) {
        const AddIn f = in[q];
        mul_fetch<K>(T, FT, f.hk, f.hv, f.hcap, f.coef, key, slot);
        __syncthreads();
        for (int e = threadIdx.x; e < G::VOL; e += blockDim.x) ACC[e] = fma(f.c, T[e], ACC[e]);
        __syncthreads();
    }
    double* dst = out.coef + (size_t)node * G::BS;
    double n2 = 0.0, w2 = 0.0;
    for (int e = threadIdx.x; e < G::BS; e += blockDim.x) {
        const int a = e % K2, b = (e / K2) % K2, c = e / (K2 * K2);
        const double v = ACC[G::at(a, b, c)];
        dst[e] = v;
        n2 += v * v;
        if (!(a < K && b < K && c < K)) w2 += v * v;
    }
    block_sum2(n2, w2, red);
    if (threadIdx.x == 0) {
        out.norm2[node] = n2;
        out.wnorm2[node] = w2;
    }
}

#define MWB_MUL_DISPATCH_K(k, F)                                                                \
    switch (k) {                                                                                \
        case 4: F(4); break;                                                                    \
        case 5: F(5); break;                                                                    \
        case 6: F(6); break;                                                                    \
        case 7: F(7); break;                                                                    \
        case 8: F(8); break;                                                                    \
        case 9: F(9); break;                                                                    \
        case 10: F(10); break;                                                                  \
        case 11: F(11); break;                                                                  \
        default: throw Error(MW_ERR_ARG, "multiply supports k = 4..11 (order 3..10)");          \
    }

namespace {

inline double mul_split_threshold(double prec, double ref, int depth) { return prec * ref * std::pow(2.0, -0.5 * depth); }

std::vector<uint64_t> host_keys(Tree& t, cudaStream_t s) {
    std::vector<uint64_t> k(t.n);
    if (t.n > 0) MWB_CUDA(cudaMemcpyAsync(k.data(), t.key, sizeof(uint64_t) * t.n, cudaMemcpyDeviceToHost, s));
    MWB_CUDA(cudaStreamSynchronize(s));
    return k;
}

// Append nodes with the given keys (zero blocks) and restore the level order (parents before
// children, keys ascending); returns the tree's keys in the new order.
std::vector<uint64_t> tree_add_keys(Tree& t, const std::vector<uint64_t>& add, cudaStream_t s) {
    if (!add.empty()) {
        const size_t BS = t.mra->bsize();
        const int n0 = t.n, na = (int)add.size();
        tree_reserve(t, n0 + na);
        MWB_CUDA(cudaMemcpyAsync(t.key + n0, add.data(), sizeof(uint64_t) * na, cudaMemcpyHostToDevice, s));
        MWB_CUDA(cudaMemsetAsync(t.coef + (size_t)n0 * BS, 0, sizeof(double) * BS * na, s));
        MWB_CUDA(cudaMemsetAsync(t.norm2 + n0, 0, sizeof(double) * na, s));
        MWB_CUDA(cudaMemsetAsync(t.wnorm2 + n0, 0, sizeof(double) * na, s));
        MWB_CUDA(cudaStreamSynchronize(s));  // `add` may leave scope
        t.n = n0 + na;
    }
    std::vector<uint64_t> keys = host_keys(t, s);
    trees_rebuild({&t}, {std::vector<char>(t.n, 1)}, {keys});
    std::sort(keys.begin(), keys.end());
    return keys;
}

std::vector<uint64_t> children_keys(uint64_t k) {
    long long tr[3];
    host_key_trans(k, tr);
    const int d = (int)(k >> 59);
    std::vector<uint64_t> c;
    for (int q = 0; q < 8; ++q)
        c.push_back(host_make_key(d + 1, 2 * tr[0] + (q & 1), 2 * tr[1] + ((q >> 1) & 1), 2 * tr[2] + ((q >> 2) & 1)));
    return c;
}

// extend the grid of `out` by the grid of `inp` (both on one world)
void build_grid(Tree& out, Tree& inp) {
    cudaStream_t s = out.mra->ctx->stream;
    if (out.n == 0) tree_make_roots(out);
    const std::vector<uint64_t> ko = host_keys(out, s), ki = host_keys(inp, s);
    std::vector<uint64_t> add;
    std::vector<uint64_t> so(ko);
    std::sort(so.begin(), so.end());
    for (uint64_t k : ki)
        if (!std::binary_search(so.begin(), so.end(), k)) add.push_back(k);
    tree_add_keys(out, add, s);
}

// split flags of the last levels of several trees in one launch: item q = (tree, node)
struct SplitTree {
    const double* wnorm2;
    const uint64_t* key;
    double thr;
};
__global__ void k_split_flags_many(const int2* __restrict__ items, int n, const SplitTree* __restrict__ ts,
                                   int depth_limit, int* flags) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int2 it = items[q];
    const SplitTree T = ts[it.x];
    flags[q] = (key_depth(T.key[it.y]) < depth_limit && sqrt(T.wnorm2[it.y]) > T.thr) ? 1 : 0;
}

// Refinement passes shared by the product and the linear combination: every pass computes the work
// nodes of all output trees with one launch (`launch(items, d_items)`), then, unless prec <= 0 or the
// pass limit is reached, splits the computed nodes whose wavelet norm exceeds prec ||out|| 2^{-depth/2}
// and makes their children the next work.  Finally every tree is compressed bottom-up with its norms.
template <typename LaunchF>
void refine_passes(double prec, int n, Tree** out, int max_iter, LaunchF&& launch) {
    const Mra* m = out[0]->mra;
    Ctx* ctx = m->ctx;
    cudaStream_t s = ctx->stream;
    // work: the current leaves of every output tree (roots for an empty tree)
    std::vector<std::vector<int>> work(n);
    std::vector<std::vector<uint64_t>> keys(n);
    std::vector<Tree*> empty;
    for (int i = 0; i < n; ++i)
        if (out[i]->n == 0) empty.push_back(out[i]);
    trees_make_roots(empty);  // all empty trees at once; their work is every root (host keys on demand)
    for (int i = 0; i < n; ++i) {
        if (std::find(empty.begin(), empty.end(), out[i]) != empty.end()) {
            for (int q = 0; q < out[i]->n; ++q) work[i].push_back(q);
            continue;
        }
        std::vector<int> c0(out[i]->n);
        MWB_CUDA(cudaMemcpyAsync(c0.data(), out[i]->child0, sizeof(int) * out[i]->n, cudaMemcpyDeviceToHost, s));
        MWB_CUDA(cudaStreamSynchronize(s));
        for (int q = 0; q < out[i]->n; ++q)
            if (c0[q] < 0) work[i].push_back(q);
        keys[i] = host_keys(*out[i], s);
    }
    for (int iter = 0;; ++iter) {
        std::vector<MulItem> items;
        for (int i = 0; i < n; ++i)
            for (int q : work[i]) items.push_back({i, q});
        if (items.empty()) break;
        MulItem* d_items = (MulItem*)dalloc(ctx, sizeof(MulItem) * items.size());
        upload_bytes(ctx, s, d_items, items.data(), sizeof(MulItem) * items.size());
        launch(items, d_items);
        MWB_CUDA(cudaGetLastError());
        ctx->launches++;
        dfree(ctx, d_items);
        if (prec <= 0.0 || (max_iter >= 0 && iter >= max_iter)) break;
        std::vector<Tree*> ts(out, out + n);
        std::vector<double> leaf2, max2;
        reduce_norms_many(ts, leaf2, max2, s);
        bool any = false;
        // trees whose work is the whole last level (always so when a tree grows from the roots): split
        // flags of all of them in one launch and one read-back, children appended as the next level
        std::vector<int> full;
        for (int i = 0; i < n; ++i) {
            const Tree& o = *out[i];
            if (work[i].empty()) continue;
            const int L = o.levels();
            const int lb = o.level_begin[L - 1], le = o.level_begin[L];
            if ((int)work[i].size() == le - lb && work[i].front() == lb && work[i].back() == le - 1) full.push_back(i);
        }
        if (!full.empty()) {
            std::vector<int2> its;
            std::vector<SplitTree> st(n, SplitTree{nullptr, nullptr, 0.0});
            for (int i : full) {
                Tree& o = *out[i];
                const int L = o.levels();
                st[i] = SplitTree{o.wnorm2, o.key, mul_split_threshold(prec, std::sqrt(leaf2[i]), L - 1)};
                for (int q = o.level_begin[L - 1]; q < o.level_begin[L]; ++q) its.push_back(int2{i, q});
            }
            const int ni = (int)its.size();
            int2* d_its = (int2*)dalloc(ctx, sizeof(int2) * ni);
            SplitTree* d_st = (SplitTree*)dalloc(ctx, sizeof(SplitTree) * n);
            int* d_flags = (int*)dalloc(ctx, sizeof(int) * ni);
            upload_bytes(ctx, s, d_its, its.data(), sizeof(int2) * ni);
            upload_bytes(ctx, s, d_st, st.data(), sizeof(SplitTree) * n);
            k_split_flags_many<<<(ni + 255) / 256, 256, 0, s>>>(d_its, ni, d_st, m->depth_limit, d_flags);
            MWB_CUDA(cudaGetLastError());
            ctx->launches++;
            std::vector<int> flags(ni);
            readback(ctx, s, {{flags.data(), d_flags, sizeof(int) * ni}});
            dfree(ctx, d_its);
            dfree(ctx, d_st);
            dfree(ctx, d_flags);
            std::vector<Tree*> grow;
            std::vector<std::vector<int>> lists;
            std::vector<int> gi;
            size_t q = 0;
            for (int i : full) {  // items are grouped by tree in `full` order
                std::vector<int> l;
                for (; q < its.size() && its[q].x == i; ++q)
                    if (flags[q]) l.push_back(its[q].y);
                work[i].clear();
                if (l.empty()) continue;
                grow.push_back(out[i]);
                lists.push_back(std::move(l));
                gi.push_back(i);
            }
            std::vector<int> before(gi.size());
            for (size_t g = 0; g < gi.size(); ++g) before[g] = out[gi[g]]->n;
            trees_add_children(grow, lists, s);
            for (size_t g = 0; g < gi.size(); ++g) {
                const int i = gi[g];
                any = true;
                for (int v = before[g]; v < out[i]->n; ++v) work[i].push_back(v);
                keys[i].clear();  // host keys are refreshed when the general path needs them
            }
        }
        for (int i = 0; i < n; ++i) {
            Tree& o = *out[i];
            if (work[i].empty() || std::find(full.begin(), full.end(), i) != full.end()) continue;
            if (keys[i].size() != (size_t)o.n) keys[i] = host_keys(o, s);
            std::vector<double> w2(o.n);
            MWB_CUDA(cudaMemcpyAsync(w2.data(), o.wnorm2, sizeof(double) * o.n, cudaMemcpyDeviceToHost, s));
            MWB_CUDA(cudaStreamSynchronize(s));
            const double ref = std::sqrt(leaf2[i]);
            std::vector<uint64_t> add;
            for (int q : work[i]) {
                const int d = (int)(keys[i][q] >> 59);
                if (d < m->depth_limit && std::sqrt(w2[q]) > mul_split_threshold(prec, ref, d)) {
                    const std::vector<uint64_t> ch = children_keys(keys[i][q]);
                    add.insert(add.end(), ch.begin(), ch.end());
                }
            }
            work[i].clear();
            if (add.empty()) continue;
            any = true;
            keys[i] = tree_add_keys(o, add, s);
            std::sort(add.begin(), add.end());
            for (uint64_t k : add)
                work[i].push_back((int)(std::lower_bound(keys[i].begin(), keys[i].end(), k) - keys[i].begin()));
        }
        if (!any) break;
    }
    trees_finish(std::vector<Tree*>(out, out + n), false, true, true, s);
    MWB_CUDA(cudaStreamSynchronize(s));
}

// out[i] = c[i] a[i] b[i], lock-step passes over the batch
void multiply_batched(double prec, int n, Tree** out, const double* c, Tree** a, Tree** b, int max_iter) {
    const Mra* m = a[0]->mra;
    Ctx* ctx = m->ctx;
    cudaStream_t s = ctx->stream;
    const int K = m->k;
    for (int i = 0; i < n; ++i) {
        if (!out[i] || !a[i] || !b[i]) throw Error(MW_ERR_ARG, "null tree");
        if (out[i]->mra != m || a[i]->mra != m || b[i]->mra != m) throw Error(MW_ERR_ARG, "trees on different worlds");
        if (a[i]->n == 0 || b[i]->n == 0) throw Error(MW_ERR_STATE, "empty input tree");
        for (int j = 0; j < n; ++j)
            if (j != i && out[j] == out[i]) throw Error(MW_ERR_ARG, "output tree listed twice");
        if (out[i] == a[i] || out[i] == b[i]) throw Error(MW_ERR_ARG, "output tree is also an input");
    }
    std::vector<MulTree> mt(n);
    MulTree* d_trees = (MulTree*)dalloc(ctx, sizeof(MulTree) * n);
    refine_passes(prec, n, out, max_iter, [&](const std::vector<MulItem>& items, const MulItem* d_items) {
        for (int i = 0; i < n; ++i) {  // output arrays may have moved (growth) since the last pass
            Tree& o = *out[i];
            mt[i] = MulTree{o.key, o.coef, o.norm2, o.wnorm2, a[i]->hkey, a[i]->hval, a[i]->hcap, a[i]->coef,
                            b[i]->hkey, b[i]->hval, b[i]->hcap, b[i]->coef, c ? c[i] : 1.0};
        }
        MWB_CUDA(cudaMemcpyAsync(d_trees, mt.data(), sizeof(MulTree) * n, cudaMemcpyHostToDevice, s));
#define L_MUL(KK)                                                                                                 \
    {                                                                                                             \
        const size_t smem = MulCfg<KK>::SMEM;                                                                     \
        MWB_CUDA(cudaFuncSetAttribute(k_mul<KK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));        \
        k_mul<KK><<<(unsigned)items.size(), kMulThreads, smem, s>>>(d_items, d_trees, m->d_MV, m->d_PF, m->d_FT, \
                                                                     m->n0);                                      \
    }
        MWB_MUL_DISPATCH_K(K, L_MUL)
#undef L_MUL
    });
    dfree(ctx, d_trees);
    MWB_CUDA(cudaStreamSynchronize(s));
}

// out = sum_i c[i] f[i] on one world
void add_trees(double prec, Tree* out, int n, const double* c, Tree** f, int max_iter) {
    if (!out || n <= 0 || !f || !c) throw Error(MW_ERR_ARG, "null tree or empty sum");
    if (n > kAddMaxTerms) throw Error(MW_ERR_ARG, "at most 256 functions per sum");
    const Mra* m = out->mra;
    Ctx* ctx = m->ctx;
    cudaStream_t s = ctx->stream;
    std::vector<AddIn> in(n);
    for (int i = 0; i < n; ++i) {
        if (!f[i]) throw Error(MW_ERR_ARG, "null tree");
        if (f[i]->mra != m) throw Error(MW_ERR_ARG, "trees on different worlds");
        if (f[i]->n == 0) throw Error(MW_ERR_STATE, "empty input tree");
        if (f[i] == out) throw Error(MW_ERR_ARG, "output tree is also an input");
        in[i] = AddIn{f[i]->hkey, f[i]->hval, f[i]->hcap, f[i]->coef, c[i]};
    }
    AddIn* d_in = (AddIn*)dalloc(ctx, sizeof(AddIn) * n);
    MWB_CUDA(cudaMemcpyAsync(d_in, in.data(), sizeof(AddIn) * n, cudaMemcpyHostToDevice, s));
    const int K = m->k;
    Tree* outs[1] = {out};
    refine_passes(prec, 1, outs, max_iter, [&](const std::vector<MulItem>& items, const MulItem* d_items) {
        const AddOut ao{out->key, out->coef, out->norm2, out->wnorm2};
#define L_ADD(KK)                                                                                                   \
    {                                                                                                               \
        const size_t smem = MulCfg<KK>::SMEM;                                                                       \
        MWB_CUDA(cudaFuncSetAttribute(k_add<KK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));          \
        k_add<KK><<<(unsigned)items.size(), kMulThreads, smem, s>>>(d_items, ao, d_in, n, m->d_FT);               \
    }
        MWB_MUL_DISPATCH_K(K, L_ADD)
#undef L_ADD
    });
    dfree(ctx, d_in);
    MWB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace
}  // namespace mwb

struct mw_tree_s : mwb::Tree {};

#define MWM_TRY(...)                                \
    try {                                           \
        __VA_ARGS__;                                \
        return MW_OK;                               \
    } catch (const mwb::Error& e) {                 \
        mwb::set_last_error(e.what());              \
        return e.code;                              \
    } catch (const std::exception& e) {             \
        mwb::set_last_error(e.what());              \
        return MW_ERR_STATE;                        \
    }
#define MWM_ARG(cond, msg) \
    if (!(cond)) throw mwb::Error(MW_ERR_ARG, msg)

extern "C" {

int mw_multiply(double prec, mw_tree out, double c, mw_tree a, mw_tree b, int max_iter) {
    MWM_TRY({
        MWM_ARG(out && a && b, "null tree");
        MWB_CUDA(cudaSetDevice(a->mra->ctx->device));
        mwb::Tree* o = out;
        mwb::Tree* pa = a;
        mwb::Tree* pb = b;
        mwb::multiply_batched(prec, 1, &o, &c, &pa, &pb, max_iter);
    })
}

int mw_multiply_batched(int n, double prec, mw_tree* out, const double* c, mw_tree* a, mw_tree* b, int max_iter) {
    MWM_TRY({
        MWM_ARG(n > 0 && out && a && b, "null pointer or empty batch");
        MWM_ARG(a[0], "null input tree");
        MWB_CUDA(cudaSetDevice(a[0]->mra->ctx->device));
        std::vector<mwb::Tree*> o(n), pa(n), pb(n);
        for (int q = 0; q < n; ++q) {
            o[q] = out[q];
            pa[q] = a[q];
            pb[q] = b[q];
        }
        mwb::multiply_batched(prec, n, o.data(), c, pa.data(), pb.data(), max_iter);
    })
}

int mw_square(double prec, mw_tree out, mw_tree a, int max_iter) { return mw_multiply(prec, out, 1.0, a, a, max_iter); }

int mw_add(double prec, mw_tree out, int n, const double* c, mw_tree* f, int max_iter) {
    MWM_TRY({
        MWM_ARG(out && f && c && n > 0, "null pointer or empty sum");
        MWB_CUDA(cudaSetDevice(out->mra->ctx->device));
        std::vector<mwb::Tree*> v(n);
        for (int q = 0; q < n; ++q) v[q] = f[q];
        mwb::add_trees(prec, out, n, c, v.data(), max_iter);
    })
}

int mw_tree_build_grid(mw_tree out, mw_tree inp) {
    MWM_TRY({
        MWM_ARG(out && inp, "null tree");
        MWM_ARG(out->mra == inp->mra, "trees on different worlds");
        MWM_ARG(out != inp, "a tree cannot extend itself");
        MWB_CUDA(cudaSetDevice(inp->mra->ctx->device));
        mwb::build_grid(*out, *inp);
    })
}

int mw_tree_clear(mw_tree t) {
    MWM_TRY({
        MWM_ARG(t, "null tree");
        t->n = 0;
        t->level_begin.clear();
        if (t->hcap > 0) mwb::launch_hash_reset(*t, t->mra->ctx->stream);
        MWB_CUDA(cudaStreamSynchronize(t->mra->ctx->stream));
    })
}

int mw_tree_copy_grid(mw_tree out, mw_tree inp) {
    const int st = mw_tree_clear(out);
    return st != MW_OK ? st : mw_tree_build_grid(out, inp);
}

}  // extern "C"
