// mw_kernels.cu -- sm_100a kernels of the MW apply: projection and two-scale transforms, norms, tree
// bookkeeping (Morton keys, hash index, splits), candidate screening, generated input nodes and the
// FP64 non-standard-form contraction.
//
// Node blocks are (2k)^3 FP64 tensors, x fastest.  In shared memory a block is stored with the
// x-pencil stride padded to 2k+1 (odd), so that pencils along every dimension are read without bank
// conflicts; each thread owns whole pencils, which makes every 1-D transform safe in place.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdio>

#include "mw_device.cuh"
#include "mw_kernels.cuh"

namespace mwb {

__global__ void k_hash_reset(uint64_t* hk, int* hv, uint32_t cap) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += gridDim.x * blockDim.x) {
        hk[i] = kEmptyKey;
        hv[i] = -1;
    }
}
// node i with key `key` into the open-addressing index (linear probing, at most cap probes)
__device__ __forceinline__ void hash_insert_one(uint64_t* hk, int* hv, uint32_t cap, uint64_t key, int i) {
    const uint32_t mask = cap - 1;
    uint32_t h = hslot(key, mask);
    for (uint32_t p = 0; p < cap; ++p) {
        unsigned long long old = atomicCAS((unsigned long long*)&hk[h], (unsigned long long)kEmptyKey,
                                           (unsigned long long)key);
        if (old == kEmptyKey || old == key) {
            hv[h] = i;
            return;
        }
        h = (h + 1) & mask;
    }
}
__global__ void k_hash_insert(uint64_t* hk, int* hv, uint32_t cap, const uint64_t* keys, int begin, int end) {
    const int i = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= end) return;
    hash_insert_one(hk, hv, cap, keys[i], i);
}

// ---------------------------------------------------------------------------------------------
// analytic functions (projection input)
// ---------------------------------------------------------------------------------------------

// hydrogen-like orbital (restated from reference src/analyticfunctions/HydrogenFunction.cpp:28-160)
__device__ inline double hydrogen(int n, int l, int m, double Z, double x, double y, double z) {
    double c = 0.0;
    if (n == 1 && l == 0) c = 2.0;
    else if (n == 2 && l == 0) c = 1.0 / (2.0 * sqrt(2.0));
    else if (n == 3 && l == 0) c = 1.0 / (9.0 * sqrt(3.0));
    else if (n == 2 && l == 1) c = 1.0 / (2.0 * sqrt(6.0));
    else if (n == 3 && l == 1) c = 1.0 / (9.0 * sqrt(6.0));
    else if (n == 3 && l == 2) c = 1.0 / (9.0 * sqrt(30.0));
    const double c0 = c * pow(Z, 1.5), c1 = 2.0 * Z / n;
    double a = 0.0;
    if (l == 0) a = 1.0;
    else if (l == 1) a = sqrt(3.0);
    else if (l == 2) a = (m <= 2) ? sqrt(15.0) : (m == 3 ? sqrt(15.0 / 4.0) : sqrt(5.0 / 4.0));
    const double ca = a / (2.0 * sqrt(3.14159265358979323846));
    const double rr = sqrt(x * x + y * y + z * z);
    const double rho = c1 * rr;
    double poly = 0.0;
    if (n == 1 && l == 0) poly = 1.0;
    else if (n == 2 && l == 0) poly = 2.0 - rho;
    else if (n == 3 && l == 0) poly = 6.0 - 6.0 * rho + rho * rho;
    else if (n == 2 && l == 1) poly = rho;
    else if (n == 3 && l == 1) poly = rho * (4.0 - rho);
    else if (n == 3 && l == 2) poly = rho * rho;
    const double radial = c0 * poly * exp(-0.5 * rho);
    double ang = 1.0;
    if (l == 1) {
        if (rr == 0.0) return 0.0;
        ang = (m == 0 ? x : (m == 1 ? y : z)) / rr;
    } else if (l == 2) {
        if (rr == 0.0) return 0.0;
        const double r2 = rr * rr;
        if (m == 0) ang = x * y / r2;
        else if (m == 1) ang = x * z / r2;
        else if (m == 2) ang = y * z / r2;
        else if (m == 3) ang = (x * x - y * y) / r2;
        else ang = (2.0 * z * z - x * x - y * y) / r2;
    }
    return radial * ca * ang;
}

__device__ inline double eval_func(const FuncDesc& f, double x, double y, double z) {
    double v = 0.0;
    if (f.type == 1) {
        for (int g = 0; g < f.nterm; ++g) {
            const double* q = f.p + 1 + 8 * g;
            const double dx = x - q[2], dy = y - q[3], dz = z - q[4];
            double p = 1.0;
            for (int i = 0; i < (int)q[5]; ++i) p *= dx;
            for (int i = 0; i < (int)q[6]; ++i) p *= dy;
            for (int i = 0; i < (int)q[7]; ++i) p *= dz;
            v += q[0] * p * exp(-q[1] * (dx * dx + dy * dy + dz * dz));
        }
    } else if (f.type == 2) {
        for (int t = 0; t < f.nterm; ++t) {
            const double* q = f.p + 1 + 11 * t;
            const double X = x - q[8], Y = y - q[9], Zc = z - q[10];
            double a = hydrogen((int)q[1], (int)q[2], (int)q[3], q[7], X, Y, Zc);
            double b = ((int)q[4] > 0) ? hydrogen((int)q[4], (int)q[5], (int)q[6], q[7], X, Y, Zc) : 1.0;
            v += q[0] * a * b;
        }
    }
    return v;
}

// ---------------------------------------------------------------------------------------------
// projection / compression / sum-up of node blocks
// ---------------------------------------------------------------------------------------------

struct TView {
    uint64_t* key;
    int* parent;
    int* child0;
    double* coef;
    double* norm2;
    double* wnorm2;
};
inline TView view(Tree& t) { return TView{t.key, t.parent, t.child0, t.coef, t.norm2, t.wnorm2}; }

struct WorldGeo {
    int n0;
    double lo[3];  // world corner (physical)
    double qx[16]; // quadrature nodes on [0,1]
};

constexpr int kTransformThreads = 256;

// one node of a transform (the whole block); leaves must have been filtered out by the caller in
// the compress / sum-up modes
template <int K>
__device__ __forceinline__ void transform_node(int mode, int node, const TView& t, const double* __restrict__ Mg,
                                               const FuncDesc& f, const WorldGeo& wg) {
    using G = Geo<K>;
    extern __shared__ double sm[];
    double* A = sm;
    double* M = A + G::VOL;
    double* red = M + G::K2 * G::K2;
    for (int i = threadIdx.x; i < G::K2 * G::K2; i += blockDim.x) M[i] = Mg[i];
    double fac = 1.0;
    if (mode == TM_PROJECT) {
        long long tr[3];
        const uint64_t key = t.key[node];
        key_trans(key, tr);
        const int n1 = wg.n0 + key_depth(key) + 1;
        const double h = ldexp(1.0, -n1);
        fac = pow(2.0, -1.5 * n1);
        for (int e = threadIdx.x; e < G::BS; e += blockDim.x) {
            const int a = e % G::K2, b = (e / G::K2) % G::K2, c = e / (G::K2 * G::K2);
            const double x = wg.lo[0] + (2 * tr[0] + a / K + wg.qx[a % K]) * h;
            const double y = wg.lo[1] + (2 * tr[1] + b / K + wg.qx[b % K]) * h;
            const double z = wg.lo[2] + (2 * tr[2] + c / K + wg.qx[c % K]) * h;
            A[G::at(a, b, c)] = eval_func(f, x, y, z);
        }
    } else if (mode == TM_COMPRESS) {
        const int c0 = t.child0[node];
        for (int e = threadIdx.x; e < G::BS; e += blockDim.x) {
            const int a = e % G::K2, b = (e / G::K2) % G::K2, c = e / (G::K2 * G::K2);
            const int ch = (a / K) + 2 * (b / K) + 4 * (c / K);
            A[G::at(a, b, c)] =
                t.coef[(size_t)(c0 + ch) * G::BS + (a % K) + G::K2 * ((b % K) + G::K2 * (c % K))];
        }
    } else {
        for (int e = threadIdx.x; e < G::BS; e += blockDim.x) {
            const int a = e % G::K2, b = (e / G::K2) % G::K2, c = e / (G::K2 * G::K2);
            A[G::at(a, b, c)] = t.coef[(size_t)node * G::BS + e];
        }
    }
    __syncthreads();
    pencil_transform<K, 0>(M, A);
    __syncthreads();
    pencil_transform<K, 1>(M, A);
    __syncthreads();
    double n2 = 0.0, w2 = 0.0;
    const int c0 = (mode == TM_SUMUP) ? t.child0[node] : 0;
    for (int p = threadIdx.x; p < G::NP; p += blockDim.x) {
        const int a = p % G::K2, b = p / G::K2;
        double x[G::K2];
#pragma unroll
        for (int i = 0; i < G::K2; ++i) x[i] = A[G::at(a, b, i)];
#pragma unroll 1
        for (int o = 0; o < G::K2; ++o) {
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < G::K2; ++i) s = fma(M[o * G::K2 + i], x[i], s);
            if (mode == TM_SUMUP) {
                const int ch = (a / K) + 2 * (b / K) + 4 * (o / K);
                t.coef[(size_t)(c0 + ch) * G::BS + (a % K) + G::K2 * ((b % K) + G::K2 * (o % K))] += s;
            } else {
                s *= fac;
                t.coef[(size_t)node * G::BS + a + G::K2 * (b + G::K2 * o)] = s;
                n2 += s * s;
                if (!(a < K && b < K && o < K)) w2 += s * s;
            }
        }
    }
    if (mode != TM_SUMUP) {
        block_sum2(n2, w2, red);
        if (threadIdx.x == 0) {
            t.norm2[node] = n2;
            t.wnorm2[node] = w2;
        }
    }
}

template <int K>
__global__ void __launch_bounds__(kTransformThreads) k_transform(int mode, const int* __restrict__ nodes, int begin,
                                                                 TView t, const double* __restrict__ Mg, FuncDesc f,
                                                                 WorldGeo wg) {
    // node list, or (nodes == nullptr) the range begin + blockIdx.x, where leaves have nothing to do
    // for the compress / sum-up modes (the whole block leaves together, before any barrier)
    const int node = nodes ? nodes[blockIdx.x] : begin + blockIdx.x;
    if (!nodes && mode != TM_PROJECT && t.child0[node] < 0) return;
    transform_node<K>(mode, node, t, Mg, f, wg);
}

// compress / sum-up of the internal nodes of one level of several trees: items (tree, node)
template <int K>
__global__ void __launch_bounds__(kTransformThreads) k_transform_multi(int mode, const int2* __restrict__ items,
                                                                       const TView* __restrict__ views,
                                                                       const double* __restrict__ Mg, WorldGeo wg) {
    const int2 it = items[blockIdx.x];
    const TView t = views[it.x];
    if (t.child0[it.y] < 0) return;
    transform_node<K>(mode, it.y, t, Mg, FuncDesc{0, 0, nullptr}, wg);
}

// one warp per (tree, node) item: squared norm of the block and of its wavelet part
template <int K>
__global__ void k_node_norms_multi(const int2* __restrict__ items, int nitems, const TView* __restrict__ views) {
    using G = Geo<K>;
    const int q = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x & 31;
    if (q >= nitems) return;
    const int2 it = items[q];
    const TView t = views[it.x];
    const double* c = t.coef + (size_t)it.y * G::BS;
    double n2 = 0.0, w2 = 0.0;
    for (int e = lane; e < G::BS; e += 32) {
        const double v = c[e];
        const int a = e % G::K2, b = (e / G::K2) % G::K2, cc = e / (G::K2 * G::K2);
        n2 += v * v;
        if (!(a < K && b < K && cc < K)) w2 += v * v;
    }
    for (int o = 16; o; o >>= 1) {
        n2 += __shfl_down_sync(0xffffffffu, n2, o);
        w2 += __shfl_down_sync(0xffffffffu, w2, o);
    }
    if (lane == 0) {
        t.norm2[it.y] = n2;
        t.wnorm2[it.y] = w2;
    }
}

// one warp per node: squared norm of the block and of its wavelet part
template <int K>
__global__ void k_node_norms(TView t, int begin, int end) {
    using G = Geo<K>;
    const int node = begin + (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x & 31;
    if (node >= end) return;
    const double* c = t.coef + (size_t)node * G::BS;
    double n2 = 0.0, w2 = 0.0;
    for (int e = lane; e < G::BS; e += 32) {
        const double v = c[e];
        const int a = e % G::K2, b = (e / G::K2) % G::K2, cc = e / (G::K2 * G::K2);
        n2 += v * v;
        if (!(a < K && b < K && cc < K)) w2 += v * v;
    }
    for (int o = 16; o; o >>= 1) {
        n2 += __shfl_down_sync(0xffffffffu, n2, o);
        w2 += __shfl_down_sync(0xffffffffu, w2, o);
    }
    if (lane == 0) {
        t.norm2[node] = n2;
        t.wnorm2[node] = w2;
    }
}

__global__ void k_split_flags(const double* __restrict__ wnorm2, const uint64_t* __restrict__ key, int begin,
                              int end, double thr, int depth_limit, int* flags) {
    const int i = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= end) return;
    flags[i - begin] = (key_depth(key[i]) < depth_limit && sqrt(wnorm2[i]) > thr) ? 1 : 0;
}
__global__ void k_internal_flags(const int* __restrict__ child0, int begin, int end, int* flags) {
    const int i = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= end) return;
    flags[i - begin] = child0[i] >= 0 ? 1 : 0;
}
__global__ void k_scatter_list(const int* __restrict__ flags, const int* __restrict__ pos, int begin, int n,
                               int* list) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (flags[i]) list[pos[i]] = begin + i;
}
__global__ void k_make_children(TView t, const int* __restrict__ list, int nsplit, int nold) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nsplit) return;
    const int p = list[q];
    const int c0 = nold + 8 * q;
    t.child0[p] = c0;
    long long tr[3];
    const uint64_t key = t.key[p];
    key_trans(key, tr);
    const int d = key_depth(key) + 1;
    for (int c = 0; c < 8; ++c) {
        const int i = c0 + c;
        t.key[i] = make_key(d, 2 * tr[0] + (c & 1), 2 * tr[1] + ((c >> 1) & 1), 2 * tr[2] + ((c >> 2) & 1));
        t.parent[i] = p;
        t.child0[i] = -1;
        t.norm2[i] = 0.0;
        t.wnorm2[i] = 0.0;
    }
}

// children of the split nodes of several trees in one launch: entry q of the flat list belongs to tree
// tree_of[q]; its 8 children are appended after the tree's first nold nodes (in list order) and
// entered into the tree's hash index
struct ChildTree {
    TView t;
    uint64_t* hkey;
    int* hval;
    uint32_t hcap;
    int nold;   // nodes before the appended children
    int first;  // first list entry of this tree
};
__global__ void k_make_children_many(const ChildTree* __restrict__ ts, const int* __restrict__ tree_of,
                                     const int* __restrict__ list, int ntot) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= ntot) return;
    const ChildTree& T = ts[tree_of[q]];
    const int p = list[q];
    const int c0 = T.nold + 8 * (q - T.first);
    T.t.child0[p] = c0;
    long long tr[3];
    const uint64_t key = T.t.key[p];
    key_trans(key, tr);
    const int d = key_depth(key) + 1;
    for (int c = 0; c < 8; ++c) {
        const int i = c0 + c;
        const uint64_t ck = make_key(d, 2 * tr[0] + (c & 1), 2 * tr[1] + ((c >> 1) & 1), 2 * tr[2] + ((c >> 2) & 1));
        T.t.key[i] = ck;
        T.t.parent[i] = p;
        T.t.child0[i] = -1;
        T.t.norm2[i] = 0.0;
        T.t.wnorm2[i] = 0.0;
        hash_insert_one(T.hkey, T.hval, T.hcap, ck, i);
    }
}

// deterministic single-block reductions (fixed summation order)
__device__ __forceinline__ double reduce_norm2_block(const double* __restrict__ norm2, const int* __restrict__ child0,
                                                     int begin, int end, int leaves_only, int want_max) {
    __shared__ double red[64];
    double s = 0.0, dummy = 0.0;
    for (int i = begin + threadIdx.x; i < end; i += blockDim.x) {
        if (leaves_only && child0[i] >= 0) continue;
        s = want_max ? fmax(s, norm2[i]) : s + norm2[i];
    }
    if (want_max) {
        for (int o = 16; o; o >>= 1) s = fmax(s, __shfl_down_sync(0xffffffffu, s, o));
        const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
        if (l == 0) red[w] = s;
        __syncthreads();
        if (w == 0) {
            s = l < (int)(blockDim.x >> 5) ? red[l] : 0.0;
            for (int o = 16; o; o >>= 1) s = fmax(s, __shfl_down_sync(0xffffffffu, s, o));
        }
    } else {
        block_sum2(s, dummy, red);
    }
    return s;
}
__global__ void k_reduce_norm2(const double* __restrict__ norm2, const int* __restrict__ child0, int begin,
                               int end, int leaves_only, int want_max, double* out) {
    const double s = reduce_norm2_block(norm2, child0, begin, end, leaves_only, want_max);
    if (threadIdx.x == 0) *out = s;
}
// both reductions of several trees in one launch: block b reduces tree b % nt, the leaf sum when
// b < nt, else the largest node norm (the same blocks as k_reduce_norm2, so the same sums)
struct NormSrc {
    const double* norm2;
    const int* child0;
    int n;
};
__global__ void k_reduce_norm2_many(const NormSrc* __restrict__ src, int nt, double* out) {
    const int t = blockIdx.x % nt, mx = blockIdx.x / nt;
    const NormSrc ns = src[t];
    const double s = reduce_norm2_block(ns.norm2, ns.child0, 0, ns.n, !mx, mx);
    if (threadIdx.x == 0) out[mx * nt + t] = s;
}

__global__ void k_rescale(double* coef, size_t n, double c) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        coef[i] *= c;
}

// per node of a: <a_node|b_node> over the wavelet part (all components at depth 0)
template <int K>
__global__ void k_dot_nodes(TView a, int na, const double* __restrict__ bcoef, const uint64_t* hk, const int* hv,
                            uint32_t hcap, double* part) {
    using G = Geo<K>;
    const int node = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x & 31;
    if (node >= na) return;
    const uint64_t key = a.key[node];
    const int j = hlookup(hk, hv, hcap, key);
    double s = 0.0;
    if (j >= 0) {
        const bool root = key_depth(key) == 0;
        const double* x = a.coef + (size_t)node * G::BS;
        const double* y = bcoef + (size_t)j * G::BS;
        for (int e = lane; e < G::BS; e += 32) {
            const int aa = e % G::K2, bb = (e / G::K2) % G::K2, cc = e / (G::K2 * G::K2);
            if (!root && aa < K && bb < K && cc < K) continue;
            s += x[e] * y[e];
        }
    }
    for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) part[node] = s;
}
// ||a - b||^2 contributions of a's nodes (one warp per node): root scaling parts and all wavelet
// parts of a - b, where b's node is missing its block counts as zero; with `only_missing` the
// nodes of a that b lacks alone (the second half of the sum, run with the roles swapped)
template <int K>
__global__ void k_diff_nodes(TView a, int na, const double* __restrict__ bcoef, const uint64_t* hk, const int* hv,
                             uint32_t hcap, int only_missing, double* part) {
    using G = Geo<K>;
    const int node = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x & 31;
    if (node >= na) return;
    const uint64_t key = a.key[node];
    const int j = hlookup(hk, hv, hcap, key);
    double s = 0.0;
    if (!(only_missing && j >= 0)) {
        const bool root = key_depth(key) == 0;
        const double* x = a.coef + (size_t)node * G::BS;
        const double* y = j >= 0 ? bcoef + (size_t)j * G::BS : nullptr;
        for (int e = lane; e < G::BS; e += 32) {
            const int aa = e % G::K2, bb = (e / G::K2) % G::K2, cc = e / (G::K2 * G::K2);
            if (!root && aa < K && bb < K && cc < K) continue;
            const double d = x[e] - (y ? y[e] : 0.0);
            s += d * d;
        }
    }
    for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) part[node] = s;
}
__global__ void k_sum_array(const double* __restrict__ v, int n, double* out) {
    __shared__ double red[64];
    double s = 0.0, d = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += v[i];
    block_sum2(s, d, red);
    if (threadIdx.x == 0) *out = s;
}

// ---------------------------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------------------------

static inline void count(Ctx* c, int n = 1) { c->launches += n; }

#define MWB_DISPATCH_K(k, F)                                    \
    switch (k) {                                                \
        case 4: F(4); break;                                    \
        case 5: F(5); break;                                    \
        case 6: F(6); break;                                    \
        case 7: F(7); break;                                    \
        case 8: F(8); break;                                    \
        case 9: F(9); break;                                    \
        case 10: F(10); break;                                  \
        case 11: F(11); break;                                  \
        case 12: F(12); break;                                  \
        default: throw Error(-1, "unsupported order (k must be 4..12)"); \
    }

static WorldGeo world_geo(const Mra& m) {
    WorldGeo g{};
    g.n0 = m.n0;
    for (int d = 0; d < 3; ++d) g.lo[d] = m.corner[d] * std::ldexp(1.0, -m.n0);
    for (int i = 0; i < m.k && i < 16; ++i) g.qx[i] = m.basis.qx[i];
    return g;
}

void launch_transform_nodes(Tree& t, int mode, const int* d_nodes, int nnodes, const FuncDesc* f, cudaStream_t s,
                            int begin) {
    if (nnodes <= 0) return;
    const Mra& m = *t.mra;
    const double* M = (mode == TM_PROJECT) ? m.d_PF : (mode == TM_COMPRESS ? m.d_F : m.d_FT);
    FuncDesc fd = f ? *f : FuncDesc{0, 0, nullptr};
    WorldGeo wg = world_geo(m);
    TView tv = view(t);
#define L_TR(KK)                                                                                      \
    {                                                                                                 \
        size_t smem = sizeof(double) * (Geo<KK>::VOL + 4 * KK * KK + 64);                            \
        MWB_CUDA(cudaFuncSetAttribute(k_transform<KK>, cudaFuncAttributeMaxDynamicSharedMemorySize,   \
                                      (int)smem));                                                    \
        k_transform<KK><<<nnodes, kTransformThreads, smem, s>>>(mode, d_nodes, begin, tv, M, fd, wg);   \
    }
    MWB_DISPATCH_K(m.k, L_TR)
#undef L_TR
    MWB_CUDA(cudaGetLastError());
    count(m.ctx);
}

// Finishing transforms of a batch of trees on one world, one launch per level for all trees:
// sum-up top-down (sumup), then compress bottom-up (compress), then the norms of every node (norms).
void trees_finish(const std::vector<Tree*>& ts, bool sumup, bool compress, bool norms, cudaStream_t s) {
    if (ts.empty()) return;
    const Mra& m = *ts[0]->mra;
    Ctx* ctx = m.ctx;
    int maxl = 0;
    for (Tree* t : ts) maxl = std::max(maxl, t->levels());
    // items grouped by level: [lvl_off[d], lvl_off[d+1]) are the nodes of depth d of every tree
    std::vector<int2> items;
    std::vector<int> lvl_off(maxl + 1, 0);
    for (int d = 0; d < maxl; ++d) {
        lvl_off[d] = (int)items.size();
        for (size_t i = 0; i < ts.size(); ++i)
            if (d < ts[i]->levels())
                for (int q = ts[i]->level_begin[d]; q < ts[i]->level_begin[d + 1]; ++q) items.push_back(int2{(int)i, q});
    }
    lvl_off[maxl] = (int)items.size();
    if (items.empty()) return;
    std::vector<TView> views;
    for (Tree* t : ts) views.push_back(view(*t));
    int2* d_items = (int2*)dalloc(ctx, sizeof(int2) * items.size());
    TView* d_views = (TView*)dalloc(ctx, sizeof(TView) * views.size());
    upload_bytes(ctx, d_items, items.data(), sizeof(int2) * items.size());
    upload_bytes(ctx, d_views, views.data(), sizeof(TView) * views.size());
    WorldGeo wg = world_geo(m);
    auto level = [&](int mode, int d) {
        const int n = lvl_off[d + 1] - lvl_off[d];
        if (n <= 0) return;
        const double* M = mode == TM_COMPRESS ? m.d_F : m.d_FT;
#define L_TRM(KK)                                                                                          \
    {                                                                                                      \
        size_t smem = sizeof(double) * (Geo<KK>::VOL + 4 * KK * KK + 64);                                 \
        MWB_CUDA(cudaFuncSetAttribute(k_transform_multi<KK>, cudaFuncAttributeMaxDynamicSharedMemorySize,  \
                                      (int)smem));                                                         \
        k_transform_multi<KK><<<n, kTransformThreads, smem, s>>>(mode, d_items + lvl_off[d], d_views, M, wg); \
    }
        MWB_DISPATCH_K(m.k, L_TRM)
#undef L_TRM
        MWB_CUDA(cudaGetLastError());
        count(ctx);
    };
    if (sumup)
        for (int d = 0; d + 1 < maxl; ++d) level(TM_SUMUP, d);
    if (compress)
        for (int d = maxl - 2; d >= 0; --d) level(TM_COMPRESS, d);
    if (norms) {
        const int n = (int)items.size();
#define L_NNM(KK) k_node_norms_multi<KK><<<(n * 32 + 255) / 256, 256, 0, s>>>(d_items, n, d_views);
        MWB_DISPATCH_K(m.k, L_NNM)
#undef L_NNM
        MWB_CUDA(cudaGetLastError());
        count(ctx);
    }
    dfree(ctx, d_items);
    dfree(ctx, d_views);
}

void launch_node_norms(Tree& t, int begin, int end, cudaStream_t s) {
    if (end <= begin) return;
    const int n = end - begin;
    TView tv = view(t);
#define L_NN(KK) k_node_norms<KK><<<(n * 32 + 255) / 256, 256, 0, s>>>(tv, begin, end);
    MWB_DISPATCH_K(t.mra->k, L_NN)
#undef L_NN
    MWB_CUDA(cudaGetLastError());
    count(t.mra->ctx);
}

void launch_hash_reset(Tree& t, cudaStream_t s) {
    k_hash_reset<<<std::min<uint32_t>((t.hcap + 255) / 256, 4096), 256, 0, s>>>(t.hkey, t.hval, t.hcap);
    MWB_CUDA(cudaGetLastError());
    count(t.mra->ctx);
}
void launch_hash_insert(Tree& t, int begin, int end, cudaStream_t s) {
    if (end <= begin) return;
    k_hash_insert<<<(end - begin + 255) / 256, 256, 0, s>>>(t.hkey, t.hval, t.hcap, t.key, begin, end);
    MWB_CUDA(cudaGetLastError());
    count(t.mra->ctx);
}

// flags -> exclusive scan -> list; returns the count (synchronises the stream)
static int compact_flags(Ctx* ctx, int* d_flags, int n, int begin, int* d_list, cudaStream_t s) {
    if (n <= 0) return 0;
    int* d_pos = (int*)dalloc(ctx, sizeof(int) * (n + 1));
    size_t tmp = 0;
    MWB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, d_flags, d_pos, n + 1, s));
    void* d_tmp = dalloc(ctx, tmp);
    MWB_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp, tmp, d_flags, d_pos, n + 1, s));
    k_scatter_list<<<(n + 255) / 256, 256, 0, s>>>(d_flags, d_pos, begin, n, d_list);
    MWB_CUDA(cudaGetLastError());
    count(ctx);
    int total = 0;
    MWB_CUDA(cudaMemcpyAsync(&total, d_pos + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    MWB_CUDA(cudaStreamSynchronize(s));
    dfree(ctx, d_tmp);
    dfree(ctx, d_pos);
    return total;
}

int launch_split(Tree& t, int begin, int end, int depth, double thr, int depth_limit, int* d_list,
                 cudaStream_t s) {
    (void)depth;
    const int n = end - begin;
    if (n <= 0) return 0;
    Ctx* ctx = t.mra->ctx;
    int* d_flags = (int*)dalloc(ctx, sizeof(int) * (n + 1));
    MWB_CUDA(cudaMemsetAsync(d_flags, 0, sizeof(int) * (n + 1), s));
    k_split_flags<<<(n + 255) / 256, 256, 0, s>>>(t.wnorm2, t.key, begin, end, thr, depth_limit, d_flags);
    MWB_CUDA(cudaGetLastError());
    count(ctx);
    int cnt = compact_flags(ctx, d_flags, n, begin, d_list, s);
    dfree(ctx, d_flags);
    return cnt;
}

int launch_internal_list(Tree& t, int begin, int end, int* d_list, cudaStream_t s) {
    const int n = end - begin;
    if (n <= 0) return 0;
    Ctx* ctx = t.mra->ctx;
    int* d_flags = (int*)dalloc(ctx, sizeof(int) * (n + 1));
    MWB_CUDA(cudaMemsetAsync(d_flags, 0, sizeof(int) * (n + 1), s));
    k_internal_flags<<<(n + 255) / 256, 256, 0, s>>>(t.child0, begin, end, d_flags);
    MWB_CUDA(cudaGetLastError());
    count(ctx);
    int cnt = compact_flags(ctx, d_flags, n, begin, d_list, s);
    dfree(ctx, d_flags);
    return cnt;
}

void trees_add_children(const std::vector<Tree*>& ts, const std::vector<std::vector<int>>& lists, cudaStream_t s) {
    size_t tot = 0;
    for (auto& l : lists) tot += l.size();
    if (tot == 0 || ts.empty()) return;
    Ctx* ctx = ts[0]->mra->ctx;
    std::vector<ChildTree> ct;
    std::vector<int> buf(2 * tot);  // list entries, then their tree (index into ct)
    size_t off = 0;
    for (size_t i = 0; i < ts.size(); ++i) {
        Tree& t = *ts[i];
        const int ns = (int)lists[i].size();
        if (ns == 0) continue;
        tree_reserve(t, t.n + 8 * ns);  // may move the arrays and grow the hash index
        ct.push_back(ChildTree{view(t), t.hkey, t.hval, t.hcap, t.n, (int)off});
        for (int q = 0; q < ns; ++q) {
            buf[off + q] = lists[i][q];
            buf[tot + off + q] = (int)ct.size() - 1;
        }
        off += ns;
    }
    int* d_buf = (int*)dalloc(ctx, sizeof(int) * buf.size());
    ChildTree* d_ct = (ChildTree*)dalloc(ctx, sizeof(ChildTree) * ct.size());
    upload_bytes(ctx, d_buf, buf.data(), sizeof(int) * buf.size());
    upload_bytes(ctx, d_ct, ct.data(), sizeof(ChildTree) * ct.size());
    k_make_children_many<<<(int)((tot + 127) / 128), 128, 0, s>>>(d_ct, d_buf + tot, d_buf, (int)tot);
    MWB_CUDA(cudaGetLastError());
    count(ctx);
    for (size_t i = 0; i < ts.size(); ++i) {
        Tree& t = *ts[i];
        const int ns = (int)lists[i].size();
        if (ns == 0) continue;
        t.n += 8 * ns;
        t.level_begin.push_back(t.n);
    }
    dfree(ctx, d_buf);  // stream-ordered; the host vectors were staged by upload_bytes
    dfree(ctx, d_ct);
}

void launch_make_children(Tree& t, const int* d_list, int nsplit, cudaStream_t s) {
    if (nsplit <= 0) return;
    k_make_children<<<(nsplit + 127) / 128, 128, 0, s>>>(view(t), d_list, nsplit, t.n);
    MWB_CUDA(cudaGetLastError());
    count(t.mra->ctx);
}

static double reduce_impl(Tree& t, int begin, int end, int leaves, int mx, cudaStream_t s) {
    if (end <= begin) return 0.0;
    Ctx* ctx = t.mra->ctx;
    double* d = (double*)dalloc(ctx, sizeof(double));
    k_reduce_norm2<<<1, 1024, 0, s>>>(t.norm2, t.child0, begin, end, leaves, mx, d);
    MWB_CUDA(cudaGetLastError());
    count(ctx);
    double h = 0.0;
    MWB_CUDA(cudaMemcpyAsync(&h, d, sizeof(double), cudaMemcpyDeviceToHost, s));
    MWB_CUDA(cudaStreamSynchronize(s));
    dfree(ctx, d);
    return h;
}
double reduce_leaf_norm2(Tree& t, cudaStream_t s) { return reduce_impl(t, 0, t.n, 1, 0, s); }

// squared norm (leaves) and largest node norm^2 of several trees with one synchronisation
void reduce_norms_many(const std::vector<Tree*>& ts, std::vector<double>& leaf2, std::vector<double>& max2,
                       cudaStream_t s) {
    const int n = (int)ts.size();
    leaf2.assign(n, 0.0);
    max2.assign(n, 0.0);
    if (n == 0) return;
    Ctx* ctx = ts[0]->mra->ctx;
    double* d = (double*)dalloc(ctx, sizeof(double) * 2 * n);
    std::vector<NormSrc> src(n);
    for (int i = 0; i < n; ++i) src[i] = NormSrc{ts[i]->norm2, ts[i]->child0, ts[i]->n};  // n = 0: zero sums
    NormSrc* d_src = (NormSrc*)dalloc(ctx, sizeof(NormSrc) * n);
    upload_bytes(ctx, d_src, src.data(), sizeof(NormSrc) * n);
    k_reduce_norm2_many<<<2 * n, 1024, 0, s>>>(d_src, n, d);
    MWB_CUDA(cudaGetLastError());
    count(ctx);
    dfree(ctx, d_src);
    std::vector<double> h(2 * n);
    readback(ctx, {{h.data(), d, sizeof(double) * 2 * n}});  // on the context's stream (= s)
    dfree(ctx, d);
    for (int i = 0; i < n; ++i) {
        leaf2[i] = h[i];
        max2[i] = h[n + i];
    }
}
double reduce_range_norm2(Tree& t, int begin, int end, cudaStream_t s) { return reduce_impl(t, begin, end, 0, 0, s); }
double reduce_max_norm2(Tree& t, cudaStream_t s) { return reduce_impl(t, 0, t.n, 0, 1, s); }

void launch_rescale(Tree& t, double c, cudaStream_t s) {
    if (t.n == 0) return;
    k_rescale<<<1024, 256, 0, s>>>(t.coef, (size_t)t.n * t.mra->bsize(), c);
    k_rescale<<<64, 256, 0, s>>>(t.norm2, (size_t)t.n, c * c);
    k_rescale<<<64, 256, 0, s>>>(t.wnorm2, (size_t)t.n, c * c);
    MWB_CUDA(cudaGetLastError());
    count(t.mra->ctx, 3);
}

double launch_dot(Tree& a, Tree& b, cudaStream_t s) {
    if (a.n == 0 || b.n == 0) return 0.0;
    Ctx* ctx = a.mra->ctx;
    double* part = (double*)dalloc(ctx, sizeof(double) * a.n);
    double* d = (double*)dalloc(ctx, sizeof(double));
    TView av = view(a);
#define L_DOT(KK) k_dot_nodes<KK><<<(a.n * 32 + 255) / 256, 256, 0, s>>>(av, a.n, b.coef, b.hkey, b.hval, b.hcap, part);
    MWB_DISPATCH_K(a.mra->k, L_DOT)
#undef L_DOT
    k_sum_array<<<1, 1024, 0, s>>>(part, a.n, d);
    MWB_CUDA(cudaGetLastError());
    count(ctx, 2);
    double h = 0.0;
    MWB_CUDA(cudaMemcpyAsync(&h, d, sizeof(double), cudaMemcpyDeviceToHost, s));
    MWB_CUDA(cudaStreamSynchronize(s));
    dfree(ctx, part);
    dfree(ctx, d);
    return h;
}

// ||a - b|| of two compressed trees on one world (any grids)
double launch_distance(Tree& a, Tree& b, cudaStream_t s) {
    Ctx* ctx = a.mra->ctx;
    const int nmax = std::max(1, std::max(a.n, b.n));
    double* part = (double*)dalloc(ctx, sizeof(double) * nmax);
    double* d = (double*)dalloc(ctx, sizeof(double) * 2);
    MWB_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * 2, s));
    TView av = view(a), bv = view(b);
    if (a.n > 0) {
#define L_DIFF(KK) k_diff_nodes<KK><<<(a.n * 32 + 255) / 256, 256, 0, s>>>(av, a.n, b.coef, b.hkey, b.hval, b.hcap, 0, part);
        MWB_DISPATCH_K(a.mra->k, L_DIFF)
#undef L_DIFF
        k_sum_array<<<1, 1024, 0, s>>>(part, a.n, d);
        count(ctx, 2);
    }
    if (b.n > 0) {
#define L_DIFF(KK) k_diff_nodes<KK><<<(b.n * 32 + 255) / 256, 256, 0, s>>>(bv, b.n, a.coef, a.hkey, a.hval, a.hcap, 1, part);
        MWB_DISPATCH_K(a.mra->k, L_DIFF)
#undef L_DIFF
        k_sum_array<<<1, 1024, 0, s>>>(part, b.n, d + 1);
        count(ctx, 2);
    }
    MWB_CUDA(cudaGetLastError());
    double h[2] = {0.0, 0.0};
    MWB_CUDA(cudaMemcpyAsync(h, d, sizeof(double) * 2, cudaMemcpyDeviceToHost, s));
    MWB_CUDA(cudaStreamSynchronize(s));
    dfree(ctx, part);
    dfree(ctx, d);
    return std::sqrt(h[0] + h[1]);
}

// dst[i] = src[perm[i]] for blocks of bs doubles
__global__ void k_gather_blocks(const double* __restrict__ src, const int* __restrict__ perm, int n, size_t bs,
                                double* __restrict__ dst) {
    const int i = blockIdx.x;
    if (i >= n) return;
    const double* a = src + (size_t)perm[i] * bs;
    double* b = dst + (size_t)i * bs;
    for (size_t e = threadIdx.x; e < bs; e += blockDim.x) b[e] = a[e];
}
void launch_gather_blocks(const double* src, const int* perm, int n, size_t bs, double* dst, cudaStream_t s) {
    if (n <= 0) return;
    k_gather_blocks<<<n, 256, 0, s>>>(src, perm, n, bs, dst);
    MWB_CUDA(cudaGetLastError());
}

// host copies of the key helpers for the driver
uint64_t host_make_key(int depth, long long tx, long long ty, long long tz) { return make_key(depth, tx, ty, tz); }

// the root level of several trees on one world, in two launches: each tree's hash index cleared
// (blockIdx.y = tree), then node i = root key i (Morton order) with no parent, no children and zero
// norms, entered into the index
struct RootTree {
    uint64_t* key;
    int* parent;
    int* child0;
    double* norm2;
    double* wnorm2;
    uint64_t* hkey;
    int* hval;
    uint32_t hcap;
};
__global__ void k_hash_reset_many(const RootTree* __restrict__ ts) {
    const RootTree T = ts[blockIdx.y];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < T.hcap; i += gridDim.x * blockDim.x) {
        T.hkey[i] = kEmptyKey;
        T.hval[i] = -1;
    }
}
__global__ void k_roots_many(const RootTree* __restrict__ ts, const uint64_t* __restrict__ rk, int nroot) {
    const RootTree T = ts[blockIdx.y];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nroot) return;
    T.key[i] = rk[i];
    T.parent[i] = -1;
    T.child0[i] = -1;
    T.norm2[i] = 0.0;
    T.wnorm2[i] = 0.0;
    hash_insert_one(T.hkey, T.hval, T.hcap, rk[i], i);
}
// every node of several trees into their (cleared) hash indices: blockIdx.y = tree
__global__ void k_hash_insert_many(const RootTree* __restrict__ ts, const int* __restrict__ n) {
    const RootTree T = ts[blockIdx.y];
    const int nn = n[blockIdx.y];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x)
        hash_insert_one(T.hkey, T.hval, T.hcap, T.key[i], i);
}
void trees_rehash(const std::vector<Tree*>& ts) {
    if (ts.empty()) return;
    Ctx* ctx = ts[0]->mra->ctx;
    cudaStream_t s = ctx->stream;
    std::vector<RootTree> rt;
    std::vector<int> n;
    uint32_t maxcap = 0;
    int maxn = 0;
    for (Tree* t : ts) {
        rt.push_back(RootTree{t->key, t->parent, t->child0, t->norm2, t->wnorm2, t->hkey, t->hval, t->hcap});
        n.push_back(t->n);
        maxcap = std::max(maxcap, t->hcap);
        maxn = std::max(maxn, t->n);
    }
    RootTree* d_rt = (RootTree*)dalloc(ctx, sizeof(RootTree) * rt.size());
    int* d_n = (int*)dalloc(ctx, sizeof(int) * n.size());
    upload_bytes(ctx, d_rt, rt.data(), sizeof(RootTree) * rt.size());
    upload_bytes(ctx, d_n, n.data(), sizeof(int) * n.size());
    const unsigned nt = (unsigned)rt.size();
    k_hash_reset_many<<<dim3(std::min<uint32_t>((maxcap + 255) / 256, 1024), nt), 256, 0, s>>>(d_rt);
    if (maxn > 0) k_hash_insert_many<<<dim3(std::min((maxn + 255) / 256, 1024), nt), 256, 0, s>>>(d_rt, d_n);
    MWB_CUDA(cudaGetLastError());
    count(ctx, maxn > 0 ? 2 : 1);
    dfree(ctx, d_rt);
    dfree(ctx, d_n);
}
void trees_make_roots(const std::vector<Tree*>& ts) {
    if (ts.empty()) return;
    const Mra& m = *ts[0]->mra;
    Ctx* ctx = m.ctx;
    cudaStream_t s = ctx->stream;
    std::vector<uint64_t> keys;
    for (int z = 0; z < m.boxes[2]; ++z)
        for (int y = 0; y < m.boxes[1]; ++y)
            for (int x = 0; x < m.boxes[0]; ++x) keys.push_back(host_make_key(0, x, y, z));
    std::sort(keys.begin(), keys.end());
    const int nroot = (int)keys.size();
    std::vector<RootTree> rt;
    uint32_t maxcap = 0;
    for (Tree* t : ts) {
        t->n = 0;
        t->level_begin.clear();
        tree_reserve(*t, nroot);
        rt.push_back(RootTree{t->key, t->parent, t->child0, t->norm2, t->wnorm2, t->hkey, t->hval, t->hcap});
        maxcap = std::max(maxcap, t->hcap);
    }
    uint64_t* d_rk = (uint64_t*)dalloc(ctx, sizeof(uint64_t) * nroot);
    RootTree* d_rt = (RootTree*)dalloc(ctx, sizeof(RootTree) * rt.size());
    upload_bytes(ctx, d_rk, keys.data(), sizeof(uint64_t) * nroot);
    upload_bytes(ctx, d_rt, rt.data(), sizeof(RootTree) * rt.size());
    const unsigned nt = (unsigned)rt.size();
    k_hash_reset_many<<<dim3(std::min<uint32_t>((maxcap + 255) / 256, 1024), nt), 256, 0, s>>>(d_rt);
    k_roots_many<<<dim3((nroot + 255) / 256, nt), 256, 0, s>>>(d_rt, d_rk, nroot);
    MWB_CUDA(cudaGetLastError());
    count(ctx, 2);
    dfree(ctx, d_rk);
    dfree(ctx, d_rt);
    for (Tree* t : ts) {
        t->n = nroot;
        t->level_begin = {0, nroot};
    }
}
void host_key_trans(uint64_t k, long long t[3]) { key_trans(k, t); }

}  // namespace mwb
