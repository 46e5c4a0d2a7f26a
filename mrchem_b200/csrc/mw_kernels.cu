// mw_kernels.cu -- sm_100a kernels of the MW apply: projection and two-scale transforms, norms, tree
// bookkeeping (Morton keys, hash index, splits), candidate screening, generated input nodes and the
// FP64 non-standard-form contraction.
//
// Node blocks are (2k)^3 FP64 tensors, x fastest.  In shared memory a block is stored with the
// x-pencil stride padded to 2k+1 (odd), so that pencils along every dimension are read without bank
// conflicts; each thread owns whole pencils, which makes every 1-D transform safe in place.
#include <cub/cub.cuh>

#include <cstdio>

#include "mw_kernels.cuh"

namespace mwb {

// ---------------------------------------------------------------------------------------------
// keys and hash index
// ---------------------------------------------------------------------------------------------

__host__ __device__ inline uint64_t spread3(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | v << 32) & 0x1f00000000ffffull;
    v = (v | v << 16) & 0x1f0000ff0000ffull;
    v = (v | v << 8) & 0x100f00f00f00f00full;
    v = (v | v << 4) & 0x10c30c30c30c30c3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
}
__host__ __device__ inline uint64_t compact3(uint64_t v) {
    v &= 0x1249249249249249ull;
    v = (v ^ (v >> 2)) & 0x10c30c30c30c30c3ull;
    v = (v ^ (v >> 4)) & 0x100f00f00f00f00full;
    v = (v ^ (v >> 8)) & 0x1f0000ff0000ffull;
    v = (v ^ (v >> 16)) & 0x1f00000000ffffull;
    v = (v ^ (v >> 32)) & 0x1fffffull;
    return v;
}
__host__ __device__ inline uint64_t make_key(int depth, long long tx, long long ty, long long tz) {
    return ((uint64_t)depth << 59) | spread3((uint64_t)tx) | (spread3((uint64_t)ty) << 1) |
           (spread3((uint64_t)tz) << 2);
}
__host__ __device__ inline int key_depth(uint64_t k) { return (int)(k >> 59); }
__host__ __device__ inline void key_trans(uint64_t k, long long t[3]) {
    uint64_t m = k & ((1ull << 57) - 1);
    t[0] = (long long)compact3(m);
    t[1] = (long long)compact3(m >> 1);
    t[2] = (long long)compact3(m >> 2);
}
__device__ inline uint32_t hslot(uint64_t k, uint32_t mask) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return (uint32_t)k & mask;
}
// linear probing; at most `cap` probes (the table is kept at most half full)
__device__ inline int hlookup(const uint64_t* hk, const int* hv, uint32_t cap, uint64_t key) {
    const uint32_t mask = cap - 1;
    uint32_t h = hslot(key, mask);
    for (uint32_t i = 0; i < cap; ++i) {
        const uint64_t s = hk[h];
        if (s == key) return hv[h];
        if (s == kEmptyKey) return -1;
        h = (h + 1) & mask;
    }
    return -1;
}

__global__ void k_hash_reset(uint64_t* hk, int* hv, uint32_t cap) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += gridDim.x * blockDim.x) {
        hk[i] = kEmptyKey;
        hv[i] = -1;
    }
}
__global__ void k_hash_insert(uint64_t* hk, int* hv, uint32_t cap, const uint64_t* keys, int begin, int end) {
    const int i = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= end) return;
    const uint64_t key = keys[i];
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

// ---------------------------------------------------------------------------------------------
// shared helpers
// ---------------------------------------------------------------------------------------------

template <int K>
struct Geo {
    static constexpr int K2 = 2 * K;
    static constexpr int P = K2 + 1;
    static constexpr int VOL = P * K2 * K2;
    static constexpr int NP = K2 * K2;
    static constexpr int BS = K2 * K2 * K2;
    __device__ static inline int at(int a, int b, int c) { return a + P * (b + K2 * c); }
};

// Sum two values over the block; the result is valid in thread 0.  `red` holds 64 doubles.
__device__ inline void block_sum2(double& a, double& b, double* red) {
    for (int o = 16; o; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const int nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (l == 0) {
        red[w] = a;
        red[32 + w] = b;
    }
    __syncthreads();
    if (w == 0) {
        a = l < nw ? red[l] : 0.0;
        b = l < nw ? red[32 + l] : 0.0;
        for (int o = 16; o; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
    }
}

// in-place 1-D transform of all pencils along DIM of a padded (2k)^3 shared tensor by the
// K2 x K2 shared matrix M (out[o] = sum_i M[o][i] in[i])
template <int K, int DIM>
__device__ inline void pencil_transform(const double* __restrict__ M, double* A) {
    using G = Geo<K>;
    for (int p = threadIdx.x; p < G::NP; p += blockDim.x) {
        const int u = p % G::K2, v = p / G::K2;
        int base, stride;
        if (DIM == 0) { base = G::P * (u + G::K2 * v); stride = 1; }
        else if (DIM == 1) { base = u + G::P * G::K2 * v; stride = G::P; }
        else { base = u + G::P * v; stride = G::P * G::K2; }
        double x[G::K2];
#pragma unroll
        for (int i = 0; i < G::K2; ++i) x[i] = A[base + i * stride];
#pragma unroll 1
        for (int o = 0; o < G::K2; ++o) {
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < G::K2; ++i) s = fma(M[o * G::K2 + i], x[i], s);
            A[base + o * stride] = s;
        }
    }
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

template <int K>
__global__ void __launch_bounds__(kTransformThreads) k_transform(int mode, const int* __restrict__ nodes, TView t, const double* __restrict__ Mg,
                            FuncDesc f, WorldGeo wg) {
    using G = Geo<K>;
    extern __shared__ double sm[];
    double* A = sm;
    double* M = A + G::VOL;
    double* red = M + G::K2 * G::K2;
    const int node = nodes[blockIdx.x];
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

// deterministic single-block reductions (fixed summation order)
__global__ void k_reduce_norm2(const double* __restrict__ norm2, const int* __restrict__ child0, int begin,
                               int end, int leaves_only, int want_max, double* out) {
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
    if (threadIdx.x == 0) *out = s;
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
__global__ void k_sum_array(const double* __restrict__ v, int n, double* out) {
    __shared__ double red[64];
    double s = 0.0, d = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += v[i];
    block_sum2(s, d, red);
    if (threadIdx.x == 0) *out = s;
}

// ---------------------------------------------------------------------------------------------
// apply: candidates, generated nodes, contraction
// ---------------------------------------------------------------------------------------------

struct CandArgs {
    const uint64_t* okey;
    int obegin, nwork, depth;
    const DeltaRec* deltas;
    int nprefix;
    InView in;
    double theta;
    long long ext[3];
    int* count;
    const int* offs;
    int* cdelta;
    int* csrc;
    uint64_t* greq_key;
    int* greq_leaf;
    int* ngreq;
};

// One warp per output node: walk the offset list in order, look up the input node at
// (depth, t_out - delta) (or its leaf ancestor: a generated input), screen with the node norm.
// Order of the kept candidates = order of the offset list (ballot compaction keeps lane order).
__global__ void k_candidates(CandArgs a, int fill) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x & 31;
    if (w >= a.nwork) return;
    long long to[3];
    key_trans(a.okey[a.obegin + w], to);
    int kept = 0;
    const int base = fill ? a.offs[w] : 0;
    for (int e0 = 0; e0 < a.nprefix; e0 += 32) {
        const int e = e0 + lane;
        int ok = 0, src = 0, leaf = -1;
        uint64_t gk = kEmptyKey;
        if (e < a.nprefix) {
            const DeltaRec de = a.deltas[e];
            long long ti[3];
            bool inside = true;
            for (int d = 0; d < 3; ++d) {
                ti[d] = to[d] - de.d[d];
                if (ti[d] < 0 || ti[d] >= a.ext[d]) inside = false;
            }
            if (inside) {
                const uint64_t key = make_key(a.depth, ti[0], ti[1], ti[2]);
                const int idx = hlookup(a.in.hkey, a.in.hval, a.in.hcap, key);
                if (idx >= 0) {
                    const double nu = sqrt(a.in.norm2[idx]);
                    if (nu > 0.0 && de.maxb * nu >= a.theta) { ok = 1; src = idx; }
                } else {
                    for (int da = a.depth - 1; da >= 0 && leaf < 0; --da) {
                        const int sh = a.depth - da;
                        leaf = hlookup(a.in.hkey, a.in.hval, a.in.hcap,
                                       make_key(da, ti[0] >> sh, ti[1] >> sh, ti[2] >> sh));
                    }
                    const double nul = leaf >= 0 ? sqrt(a.in.norm2[leaf]) : 0.0;
                    if (nul > 0.0 && de.maxb * nul >= a.theta) {
                        ok = 1;
                        gk = key;
                    }
                }
            }
        }
        const unsigned bal = __ballot_sync(0xffffffffu, ok);
        if (fill && ok) {
            const int pos = base + kept + __popc(bal & ((1u << lane) - 1u));
            a.cdelta[pos] = e;
            if (gk != kEmptyKey) {
                const int r = atomicAdd(a.ngreq, 1);
                a.greq_key[r] = gk;
                a.greq_leaf[r] = leaf;
                a.csrc[pos] = -(r + 1);
            } else {
                a.csrc[pos] = src;
            }
        }
        kept += __popc(bal);
    }
    if (!fill && lane == 0) a.count[w] = kept;
}

__global__ void k_unique_flags(const uint64_t* __restrict__ k, int n, int* flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    flags[i] = (i == 0 || k[i] != k[i - 1]) ? 1 : 0;
}
__global__ void k_unique_scatter(const uint64_t* __restrict__ k, const int* __restrict__ leaf,
                                 const int* __restrict__ flags, const int* __restrict__ pos, int n,
                                 uint64_t* uk, int* ul) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (flags[i]) {
        uk[pos[i]] = k[i];
        ul[pos[i]] = leaf[i];
    }
}
// replace request ids in csrc by generated-node ids (binary search in the sorted unique keys)
__global__ void k_resolve_gen(int* csrc, int ncand, const uint64_t* __restrict__ greq_key,
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

// Scaling-only block of a generated input node: reconstruct the leaf ancestor's block to its
// children, take the child on the path, then descend with zero wavelets (s_c = H_c^T s per dim).
template <int K>
__global__ void __launch_bounds__(kTransformThreads) k_generate(const uint64_t* __restrict__ ukey, const int* __restrict__ uleaf, InView in,
                           const uint64_t* __restrict__ inkey, const double* __restrict__ FT, double* gblk,
                           double* gnorm2) {
    using G = Geo<K>;
    extern __shared__ double sm[];
    double* A = sm;
    double* M = A + G::VOL;
    double* S = M + G::K2 * G::K2;
    double* red = S + K * K * K;
    const int g = blockIdx.x;
    const int leaf = uleaf[g];
    const uint64_t key = ukey[g];
    for (int i = threadIdx.x; i < G::K2 * G::K2; i += blockDim.x) M[i] = FT[i];
    for (int e = threadIdx.x; e < G::BS; e += blockDim.x) {
        const int a = e % G::K2, b = (e / G::K2) % G::K2, c = e / (G::K2 * G::K2);
        A[G::at(a, b, c)] = in.coef[(size_t)leaf * G::BS + e];
    }
    __syncthreads();
    pencil_transform<K, 0>(M, A);
    __syncthreads();
    pencil_transform<K, 1>(M, A);
    __syncthreads();
    pencil_transform<K, 2>(M, A);
    __syncthreads();
    long long t[3], tl[3];
    key_trans(key, t);
    key_trans(inkey[leaf], tl);
    const int d = key_depth(key), dl = d - key_depth(inkey[leaf]);
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
                int base, stride;
                if (dim == 0) { base = K * (u + K * v); stride = 1; }
                else if (dim == 1) { base = u + K * K * v; stride = K; }
                else { base = u + K * v; stride = K * K; }
                double x[K];
#pragma unroll
                for (int i = 0; i < K; ++i) x[i] = S[base + i * stride];
#pragma unroll 1
                for (int o = 0; o < K; ++o) {
                    double s = 0.0;
#pragma unroll
                    for (int i = 0; i < K; ++i) s = fma(M[(c * K + o) * G::K2 + i], x[i], s);
                    S[base + o * stride] = s;
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

struct ApplyArgs {
    int obegin, nwork;
    const int* coff;
    const int* cdelta;
    const int* csrc;
    const DeltaRec* deltas;
    const TermRec* terms;
    const double* mats;
    InView in;
    const double* gblk;
    const double* gnorm2;
    double theta;
    int root;
    double* ocoef;
    double* onorm2;
    double* ownorm2;
    unsigned long long* ntrip;
};

template <int K>
struct ApplyCfg {
    static constexpr int K2 = 2 * K;
    static constexpr int NP = K2 * K2;
    static constexpr bool STAGE = K2 <= 20;         // input block staged in shared memory
    static constexpr int PPT = K2 <= 20 ? 1 : 2;     // z-pencils (accumulators) per thread
    static constexpr int NT = ((NP + PPT - 1) / PPT + 31) / 32 * 32;
    static constexpr int XS = STAGE ? Geo<K>::VOL : K * K * K;
    static constexpr size_t SMEM = sizeof(double) * (size_t)(XS + Geo<K>::VOL + 3 * NP + K * K * K + 64);
};

// input element (a, b, c) of the current candidate: staged padded tensor, compact k^3 generated
// block in shared memory, or (large k, full block) straight from global memory
template <int K, bool GEN>
__device__ inline double xin(const double* X, const double* __restrict__ blk, int a, int b, int c) {
    using C = ApplyCfg<K>;
    if (C::STAGE) return X[Geo<K>::at(a, b, c)];
    if (GEN) return X[a + K * (b + K * c)];
    return __ldg(&blk[a + 2 * K * (b + 2 * K * c)]);
}

// x-step: T[:, b, c] = M_x X[:, b, c] (GEN: only the k scaling inputs, b, c < k), plus for depth > 0
// the scaling-only chain U = T_x X_sss
template <int K, bool GEN>
__device__ inline void apply_step_x(const double* __restrict__ Mx, const double* X, const double* __restrict__ blk,
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

// y-step in place on T (GEN: inputs b < k, planes c < k) and on U
template <int K, bool GEN>
__device__ inline void apply_step_y(const double* __restrict__ My, double* T, double* U, bool root) {
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

// z-step into the register accumulators of the thread's z-pencils
template <int K, bool GEN>
__device__ inline void apply_step_z(const double* __restrict__ Mz, const double* T, const double* U, bool root,
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

// FP64 NS-form contraction.  One CTA per output node; its candidates (input node, offset) and, per
// offset, the terms (sorted by bound) that pass the screening.  For every term:
//   out += beta * (NS_z (x) NS_y (x) NS_x) in       (three in-place pencil transforms)
//   out_sss -= beta * (T_z (x) T_y (x) T_x) in_sss  (depth > 0: the s->s block belongs to coarser scales)
// Accumulators live in registers (each thread owns whole z-pencils).
template <int K>
__global__ void __launch_bounds__(ApplyCfg<K>::NT, 1) k_apply_fp64(ApplyArgs A) {
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
    const int node = A.obegin + blockIdx.x;
    const int tid = threadIdx.x;
    const bool root = A.root != 0;
    double acc[C::PPT][K2];
#pragma unroll
    for (int j = 0; j < C::PPT; ++j)
#pragma unroll
        for (int c = 0; c < K2; ++c) acc[j][c] = 0.0;
    unsigned long long ntrip = 0;
    const int cb = A.coff[blockIdx.x], ce = A.coff[blockIdx.x + 1];
    for (int ci = cb; ci < ce; ++ci) {
        const int e = A.cdelta[ci];
        const int src = A.csrc[ci];
        const bool gen = src < 0;
        const double nu = gen ? sqrt(A.gnorm2[-src - 1]) : sqrt(A.in.norm2[src]);
        const DeltaRec de = A.deltas[e];
        if (!(nu > 0.0) || de.maxb * nu < A.theta) continue;
        if (A.terms[de.t0].bound * nu < A.theta) continue;
        const double* blk = gen ? A.gblk + (size_t)(-src - 1) * K * K * K : A.in.coef + (size_t)src * G::BS;
        // stage the input block (full (2k)^3, or the k^3 scaling block of a generated node); the
        // barrier keeps the previous candidate's readers and writers of X/T/U/M behind us
        __syncthreads();
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
            const TermRec tr = A.terms[ti];
            if (tr.bound * nu < A.theta) break;
            __syncthreads();
            for (int i = tid; i < C::NP; i += blockDim.x) {
                Mx[i] = A.mats[(size_t)tr.mx * C::NP + i];
                My[i] = A.mats[(size_t)tr.my * C::NP + i];
                Mz[i] = A.mats[(size_t)tr.mz * C::NP + i];
            }
            __syncthreads();
            if (gen) apply_step_x<K, true>(Mx, X, blk, T, U, root);
            else apply_step_x<K, false>(Mx, X, blk, T, U, root);
            __syncthreads();
            if (gen) apply_step_y<K, true>(My, T, U, root);
            else apply_step_y<K, false>(My, T, U, root);
            __syncthreads();
            if (gen) apply_step_z<K, true>(Mz, T, U, root, tr.beta, acc);
            else apply_step_z<K, false>(Mz, T, U, root, tr.beta, acc);
            ++ntrip;
        }
    }
    // write the NS block, its norm and its wavelet norm
    double n2 = 0.0, w2 = 0.0;
#pragma unroll
    for (int j = 0; j < C::PPT; ++j) {
        const int p = tid + j * C::NT;
        if (p < C::NP) {
            const int a = p % K2, b = p / K2;
#pragma unroll
            for (int c = 0; c < K2; ++c) {
                const double v = acc[j][c];
                A.ocoef[(size_t)node * G::BS + a + K2 * (b + K2 * c)] = v;
                n2 += v * v;
                if (!(a < K && b < K && c < K)) w2 += v * v;
            }
        }
    }
    block_sum2(n2, w2, red);
    if (tid == 0) {
        A.onorm2[node] = n2;
        A.ownorm2[node] = w2;
        atomicAdd(A.ntrip, ntrip);
    }
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

static int threads_for(int K) {
    int np = 4 * K * K;
    int nt = ((np + 31) / 32) * 32;
    return nt > 1024 ? 1024 : nt;
}

static WorldGeo world_geo(const Mra& m) {
    WorldGeo g{};
    g.n0 = m.n0;
    for (int d = 0; d < 3; ++d) g.lo[d] = m.corner[d] * std::ldexp(1.0, -m.n0);
    for (int i = 0; i < m.k && i < 16; ++i) g.qx[i] = m.basis.qx[i];
    return g;
}

void launch_transform_nodes(Tree& t, int mode, const int* d_nodes, int nnodes, const FuncDesc* f,
                            cudaStream_t s) {
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
        k_transform<KK><<<nnodes, kTransformThreads, smem, s>>>(mode, d_nodes, tv, M, fd, wg);          \
    }
    MWB_DISPATCH_K(m.k, L_TR)
#undef L_TR
    MWB_CUDA(cudaGetLastError());
    count(m.ctx);
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

void run_apply_pass(Tree& out, int obegin, int oend, Tree& inp, ApplyPass& pass, cudaStream_t s) {
    const int nwork = oend - obegin;
    if (nwork <= 0) return;
    Ctx* ctx = out.mra->ctx;
    const int K = out.mra->k;
    const OpDepth& tab = *pass.tab;
    InView in{inp.hkey, inp.hval, inp.hcap, inp.coef, inp.norm2};

    int* d_count = (int*)dalloc(ctx, sizeof(int) * (nwork + 1));
    int* d_offs = (int*)dalloc(ctx, sizeof(int) * (nwork + 1));
    int* d_ngreq = (int*)dalloc(ctx, sizeof(int));
    MWB_CUDA(cudaMemsetAsync(d_count, 0, sizeof(int) * (nwork + 1), s));
    MWB_CUDA(cudaMemsetAsync(d_ngreq, 0, sizeof(int), s));
    CandArgs ca{};
    ca.okey = out.key;
    ca.obegin = obegin;
    ca.nwork = nwork;
    ca.depth = pass.depth;
    ca.deltas = tab.d_deltas;
    ca.nprefix = pass.nprefix;
    ca.in = in;
    ca.theta = pass.theta;
    for (int d = 0; d < 3; ++d) ca.ext[d] = pass.ext[d];
    ca.count = d_count;
    const int cblocks = (nwork * 32 + 255) / 256;
    k_candidates<<<cblocks, 256, 0, s>>>(ca, 0);
    MWB_CUDA(cudaGetLastError());
    count(ctx);
    size_t tmp = 0;
    MWB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, d_count, d_offs, nwork + 1, s));
    void* d_tmp = dalloc(ctx, tmp);
    MWB_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp, tmp, d_count, d_offs, nwork + 1, s));
    int ncand = 0;
    MWB_CUDA(cudaMemcpyAsync(&ncand, d_offs + nwork, sizeof(int), cudaMemcpyDeviceToHost, s));
    MWB_CUDA(cudaStreamSynchronize(s));
    dfree(ctx, d_tmp);

    const int ncap = ncand > 0 ? ncand : 1;
    int* d_cdelta = (int*)dalloc(ctx, sizeof(int) * ncap);
    int* d_csrc = (int*)dalloc(ctx, sizeof(int) * ncap);
    uint64_t* d_greq_key = (uint64_t*)dalloc(ctx, sizeof(uint64_t) * ncap);
    int* d_greq_leaf = (int*)dalloc(ctx, sizeof(int) * ncap);
    ca.offs = d_offs;
    ca.cdelta = d_cdelta;
    ca.csrc = d_csrc;
    ca.greq_key = d_greq_key;
    ca.greq_leaf = d_greq_leaf;
    ca.ngreq = d_ngreq;
    if (ncand > 0) {
        k_candidates<<<cblocks, 256, 0, s>>>(ca, 1);
        MWB_CUDA(cudaGetLastError());
        count(ctx);
    }
    int ngreq = 0;
    MWB_CUDA(cudaMemcpyAsync(&ngreq, d_ngreq, sizeof(int), cudaMemcpyDeviceToHost, s));
    MWB_CUDA(cudaStreamSynchronize(s));

    // generated input nodes: sort the requests by key, keep one per key, resolve candidate ids
    int nu = 0;
    uint64_t* d_ukey = nullptr;
    int* d_uleaf = nullptr;
    double* d_gblk = nullptr;
    double* d_gnorm2 = nullptr;
    if (ngreq > 0) {
        uint64_t* d_sk = (uint64_t*)dalloc(ctx, sizeof(uint64_t) * ngreq);
        int* d_sl = (int*)dalloc(ctx, sizeof(int) * ngreq);
        tmp = 0;
        MWB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, d_greq_key, d_sk, d_greq_leaf, d_sl, ngreq, 0, 64, s));
        d_tmp = dalloc(ctx, tmp);
        MWB_CUDA(cub::DeviceRadixSort::SortPairs(d_tmp, tmp, d_greq_key, d_sk, d_greq_leaf, d_sl, ngreq, 0, 64, s));
        dfree(ctx, d_tmp);
        int* d_flags = (int*)dalloc(ctx, sizeof(int) * (ngreq + 1));
        int* d_pos = (int*)dalloc(ctx, sizeof(int) * (ngreq + 1));
        MWB_CUDA(cudaMemsetAsync(d_flags, 0, sizeof(int) * (ngreq + 1), s));
        k_unique_flags<<<(ngreq + 255) / 256, 256, 0, s>>>(d_sk, ngreq, d_flags);
        tmp = 0;
        MWB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, d_flags, d_pos, ngreq + 1, s));
        d_tmp = dalloc(ctx, tmp);
        MWB_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp, tmp, d_flags, d_pos, ngreq + 1, s));
        dfree(ctx, d_tmp);
        MWB_CUDA(cudaMemcpyAsync(&nu, d_pos + ngreq, sizeof(int), cudaMemcpyDeviceToHost, s));
        MWB_CUDA(cudaStreamSynchronize(s));
        d_ukey = (uint64_t*)dalloc(ctx, sizeof(uint64_t) * nu);
        d_uleaf = (int*)dalloc(ctx, sizeof(int) * nu);
        k_unique_scatter<<<(ngreq + 255) / 256, 256, 0, s>>>(d_sk, d_sl, d_flags, d_pos, ngreq, d_ukey, d_uleaf);
        k_resolve_gen<<<(ncand + 255) / 256, 256, 0, s>>>(d_csrc, ncand, d_greq_key, d_ukey, nu);
        MWB_CUDA(cudaGetLastError());
        d_gblk = (double*)dalloc(ctx, sizeof(double) * (size_t)nu * K * K * K);
        d_gnorm2 = (double*)dalloc(ctx, sizeof(double) * nu);
#define L_GEN(KK)                                                                                      \
    {                                                                                                  \
        size_t smem = sizeof(double) * (Geo<KK>::VOL + 4 * KK * KK + KK * KK * KK + 64);              \
        MWB_CUDA(cudaFuncSetAttribute(k_generate<KK>, cudaFuncAttributeMaxDynamicSharedMemorySize,     \
                                      (int)smem));                                                     \
        k_generate<KK><<<nu, kTransformThreads, smem, s>>>(d_ukey, d_uleaf, in, inp.key, out.mra->d_FT,  \
                                                         d_gblk, d_gnorm2);                            \
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

    unsigned long long* d_ntrip = (unsigned long long*)dalloc(ctx, sizeof(unsigned long long));
    MWB_CUDA(cudaMemsetAsync(d_ntrip, 0, sizeof(unsigned long long), s));
    ApplyArgs aa{};
    aa.obegin = obegin;
    aa.nwork = nwork;
    aa.coff = d_offs;
    aa.cdelta = d_cdelta;
    aa.csrc = d_csrc;
    aa.deltas = tab.d_deltas;
    aa.terms = tab.d_terms;
    aa.mats = tab.d_mats;
    aa.in = in;
    aa.gblk = d_gblk;
    aa.gnorm2 = d_gnorm2;
    aa.theta = pass.theta;
    aa.root = pass.root ? 1 : 0;
    aa.ocoef = out.coef;
    aa.onorm2 = out.norm2;
    aa.ownorm2 = out.wnorm2;
    aa.ntrip = d_ntrip;
#define L_AP(KK)                                                                                      \
    {                                                                                                 \
        size_t smem = ApplyCfg<KK>::SMEM;                                                             \
        MWB_CUDA(cudaFuncSetAttribute(k_apply_fp64<KK>, cudaFuncAttributeMaxDynamicSharedMemorySize,  \
                                      (int)smem));                                                    \
        k_apply_fp64<KK><<<nwork, ApplyCfg<KK>::NT, smem, s>>>(aa);                                   \
    }
    if (ctx->prof) MWB_CUDA(cudaEventRecord(ctx->ev0, s));
    MWB_DISPATCH_K(K, L_AP)
#undef L_AP
    MWB_CUDA(cudaGetLastError());
    if (ctx->prof) MWB_CUDA(cudaEventRecord(ctx->ev1, s));
    count(ctx);
    ctx->apply_launches++;
    unsigned long long nt = 0;
    MWB_CUDA(cudaMemcpyAsync(&nt, d_ntrip, sizeof(nt), cudaMemcpyDeviceToHost, s));
    MWB_CUDA(cudaStreamSynchronize(s));
    if (ctx->prof) {
        float ms = 0.0f;
        MWB_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        ctx->apply_ms += ms;
    }
    pass.triples = (long long)nt;
    pass.triples_gen = 0;

    dfree(ctx, d_ntrip);
    if (d_gblk) dfree(ctx, d_gblk);
    if (d_gnorm2) dfree(ctx, d_gnorm2);
    if (d_ukey) dfree(ctx, d_ukey);
    if (d_uleaf) dfree(ctx, d_uleaf);
    dfree(ctx, d_cdelta);
    dfree(ctx, d_csrc);
    dfree(ctx, d_greq_key);
    dfree(ctx, d_greq_leaf);
    dfree(ctx, d_count);
    dfree(ctx, d_offs);
    dfree(ctx, d_ngreq);
}

// host copies of the key helpers for the driver
uint64_t host_make_key(int depth, long long tx, long long ty, long long tz) { return make_key(depth, tx, ty, tz); }
void host_key_trans(uint64_t k, long long t[3]) { key_trans(k, t); }

}  // namespace mwb
