// mw_learned.cu -- learned output-tree proposal for the adaptive apply.
//
// A small MLP (FP32, 3 hidden layers of 128 by default) predicts, for a candidate output node, whether
// the plain wavelet-norm check will split it.  Its 64 features are: level, position, the block and
// wavelet norms of the 27 input neighbours at the node's depth (relative to the split threshold),
// and operator / precision scales.  It is trained on the GPU by the kernels below (forward, backward,
// Adam) from labels produced by plain applies.
//
// The learned apply (apply_learned) runs the exact root pass, proposes the whole deeper tree with
// the network, computes every proposed node in one batched pass, then applies the plain criterion
// top-down to every computed node: proposed nodes the criterion would not have created are pruned,
// and nodes the criterion splits but the network did not are refined with further passes.  The
// result is the plain apply's tree (node keys and coefficients) exactly.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <numeric>
#include <random>
#include <unordered_map>

#include "../../include/mwb200.h"
#include "mw_device.cuh"
#include "mw_kernels.cuh"
#include "mw_learned.cuh"

namespace mwb {

void set_last_error(const std::string& msg);

// ---------------------------------------------------------------------------------------------
// features
// ---------------------------------------------------------------------------------------------
struct FeatTree {
    const uint64_t* okey;   // output tree keys
    const uint64_t* ikey;   // input tree keys
    const double* inorm2;   // input block norms^2
    const double* iwnorm2;  // input wavelet norms^2
    const uint64_t* hkey;
    const int* hval;
    uint32_t hcap;
    const double* owind2;   // output wavelet norms^2 (the root nodes' are exact after the root pass)
    const uint64_t* ohkey;  // output hash index (root lookup)
    const int* ohval;
    uint32_t ohcap;
    int n0;
    int boxes[3];
    double thr0;            // split threshold at depth 0 (prec * g0)
    double mu, prec;
};

__device__ inline float lg(double v) { return (float)(log10(v + 1e-30) * 0.1); }

// one thread per (entry, node): writes kNF features
// One warp per candidate node: lane j < 27 takes neighbour j (dz, dy, dx in -1..1, dx fastest), lane 27
// the node's own features; the neighbours' hash probes and ancestor walks run side by side
__global__ void k_features(const int2* __restrict__ items, int n, const FeatTree* __restrict__ trees, float* F) {
    const int i = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= n || lane > 27) return;
    const int2 it = items[i];
    const FeatTree& T = trees[it.x];
    const uint64_t key = T.okey[it.y];
    const int d = key_depth(key);
    long long t[3];
    key_trans(key, t);
    const double thr = T.thr0 * pow(2.0, -0.5 * d);
    float* f = F + (size_t)i * kNF;
    if (lane < 27) {
        const int dx = lane % 3 - 1, dy = (lane / 3) % 3 - 1, dz = lane / 9 - 1;
        const long long u[3] = {t[0] + dx, t[1] + dy, t[2] + dz};
        bool inside = true;
        for (int q = 0; q < 3; ++q) inside &= u[q] >= 0 && u[q] < ((long long)T.boxes[q] << d);
        float fb = -3.0f, fw = -3.0f;
        if (inside) {
            int idx = hlookup(T.hkey, T.hval, T.hcap, make_key(d, u[0], u[1], u[2]));
            if (idx >= 0) {
                fb = lg(sqrt(T.inorm2[idx]) / thr);
                fw = lg(sqrt(T.iwnorm2[idx]) / thr);
            } else {
                for (int da = d - 1; da >= 0 && idx < 0; --da) {
                    const int sh = d - da;
                    idx = hlookup(T.hkey, T.hval, T.hcap, make_key(da, u[0] >> sh, u[1] >> sh, u[2] >> sh));
                    if (idx >= 0) fb = lg(sqrt(T.inorm2[idx]) * pow(2.0, -1.5 * sh) / thr);
                }
            }
        }
        f[4 + 2 * lane] = fb;
        f[5 + 2 * lane] = fw;
        return;
    }
    f[0] = d / 16.0f;
    for (int q = 0; q < 3; ++q) f[1 + q] = (float)(2.0 * (t[q] + 0.5) / ((double)T.boxes[q] * (1ll << d)) - 1.0);
    f[58] = (float)log10(T.mu + 1e-3);
    f[59] = (float)(log10(T.prec) * 0.1);
    const double edge = ldexp(1.0, -(T.n0 + d));
    f[60] = (float)log10(edge);
    f[61] = (float)log10(T.mu * edge + 1e-3);
    f[62] = lg(thr);
    const int r = hlookup(T.ohkey, T.ohval, T.ohcap, make_key(0, t[0] >> d, t[1] >> d, t[2] >> d));
    f[63] = r >= 0 ? lg(sqrt(T.owind2[r]) / T.thr0) : 0.0f;
}

// ---------------------------------------------------------------------------------------------
// MLP kernels (FP32)
// ---------------------------------------------------------------------------------------------
// Y[n][o] = act(sum_i X[n][i] W[o][i] + b[o]); 16x16 tiles
__global__ void k_lin_fwd(const float* __restrict__ X, const float* __restrict__ W, const float* __restrict__ b, float* Y,
                          int N, int in, int out, int relu) {
    __shared__ float xs[16][17], ws[16][17];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int n = blockIdx.x * 16 + ty, o = blockIdx.y * 16 + tx;
    float acc = 0.0f;
    for (int k0 = 0; k0 < in; k0 += 16) {
        xs[ty][tx] = (n < N && k0 + tx < in) ? X[(size_t)n * in + k0 + tx] : 0.0f;
        const int ow = blockIdx.y * 16 + ty;
        ws[ty][tx] = (ow < out && k0 + tx < in) ? W[(size_t)ow * in + k0 + tx] : 0.0f;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 16; ++k) acc = fmaf(xs[ty][k], ws[tx][k], acc);
        __syncthreads();
    }
    if (n < N && o < out) {
        float v = acc + b[o];
        Y[(size_t)n * out + o] = (relu && v < 0.0f) ? 0.0f : v;
    }
}
// dX[n][i] = sum_o dY[n][o] W[o][i] (dY already masked by the activation)
__global__ void k_lin_bwd_x(const float* __restrict__ dY, const float* __restrict__ W, float* dX, int N, int in, int out) {
    __shared__ float ds[16][17], ws[16][17];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int n = blockIdx.x * 16 + ty, i = blockIdx.y * 16 + tx;
    float acc = 0.0f;
    for (int o0 = 0; o0 < out; o0 += 16) {
        ds[ty][tx] = (n < N && o0 + tx < out) ? dY[(size_t)n * out + o0 + tx] : 0.0f;
        ws[ty][tx] = (o0 + ty < out && i < in) ? W[(size_t)(o0 + ty) * in + i] : 0.0f;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 16; ++k) acc = fmaf(ds[ty][k], ws[k][tx], acc);
        __syncthreads();
    }
    if (n < N && i < in) dX[(size_t)n * in + i] = acc;
}
// dW[o][i] = sum_n dY[n][o] X[n][i]; db[o] = sum_n dY[n][o] (one block per 16x16 tile, fixed order)
__global__ void k_lin_bwd_w(const float* __restrict__ dY, const float* __restrict__ X, float* dW, float* db, int N,
                            int in, int out) {
    __shared__ float ds[16][17], xs[16][17];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int o = blockIdx.y * 16 + ty, i = blockIdx.x * 16 + tx;
    float acc = 0.0f, accb = 0.0f;
    for (int n0 = 0; n0 < N; n0 += 16) {
        ds[ty][tx] = (n0 + tx < N && blockIdx.y * 16 + ty < out) ? dY[(size_t)(n0 + tx) * out + blockIdx.y * 16 + ty] : 0.0f;
        xs[ty][tx] = (n0 + ty < N && i < in) ? X[(size_t)(n0 + ty) * in + i] : 0.0f;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            acc = fmaf(ds[ty][k], xs[k][tx], acc);
            accb += ds[ty][k];
        }
        __syncthreads();
    }
    if (o < out && i < in) dW[(size_t)o * in + i] = acc;
    if (o < out && blockIdx.x == 0 && tx == 0) db[o] = accb;
}
__global__ void k_relu_mask(float* dY, const float* __restrict__ Y, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        if (Y[i] <= 0.0f) dY[i] = 0.0f;
}
// weighted BCE with logits: loss_i = w_i (softplus(z) - y z); dz_i = w_i (sigmoid(z) - y) / N
__global__ void k_bce(const float* __restrict__ z, const float* __restrict__ y, const float* __restrict__ w, int N,
                      float* dz, float* loss_part) {
    __shared__ float red[32];
    float l = 0.0f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const float zi = z[i];
        const float sp = zi > 0.0f ? zi + log1pf(expf(-zi)) : log1pf(expf(zi));
        l += w[i] * (sp - y[i] * zi);
        const float sg = 1.0f / (1.0f + expf(-zi));
        dz[i] = w[i] * (sg - y[i]) / (float)N;
    }
    for (int o = 16; o; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x < 32) {
        l = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0f;
        for (int o = 16; o; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
        if (threadIdx.x == 0) loss_part[blockIdx.x] = l;
    }
}
__global__ void k_adam(float* p, const float* __restrict__ g, float* m, float* v, int n, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    m[i] = b1 * m[i] + (1.0f - b1) * gi;
    v[i] = b2 * v[i] + (1.0f - b2) * gi * gi;
    p[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
}
__global__ void k_gather_rows(const float* __restrict__ src, const int* __restrict__ idx, int n, int w, float* dst) {
    const int i = blockIdx.x;
    if (i >= n) return;
    for (int j = threadIdx.x; j < w; j += blockDim.x) dst[(size_t)i * w + j] = src[(size_t)idx[i] * w + j];
}

// ---------------------------------------------------------------------------------------------
// MLP object
// ---------------------------------------------------------------------------------------------
Mlp::~Mlp() {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    for (float* q : {d_p, d_m, d_v, d_g, d_X, d_y}) dfree(ctx, q);
    cudaStreamSynchronize(ctx->stream);
}

void mlp_init(Mlp& M, Ctx* ctx, int nhidden, int width, unsigned seed) {
    M.ctx = ctx;
    M.nhidden = nhidden;
    M.width = width;
    M.dims = {kNF};
    for (int l = 0; l < nhidden; ++l) M.dims.push_back(width);
    M.dims.push_back(1);
    M.nparam = 0;
    for (size_t l = 0; l + 1 < M.dims.size(); ++l) {
        M.woff.push_back(M.nparam);
        M.nparam += (size_t)M.dims[l] * M.dims[l + 1];
        M.boff.push_back(M.nparam);
        M.nparam += M.dims[l + 1];
    }
    std::vector<float> p(M.nparam, 0.0f);
    std::mt19937 rng(seed);
    for (size_t l = 0; l + 1 < M.dims.size(); ++l) {
        std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / M.dims[l]));  // He initialisation
        for (size_t q = 0; q < (size_t)M.dims[l] * M.dims[l + 1]; ++q) p[M.woff[l] + q] = nd(rng);
    }
    cudaStream_t s = ctx->stream;
    M.d_p = (float*)dalloc(ctx, sizeof(float) * M.nparam);
    M.d_m = (float*)dalloc(ctx, sizeof(float) * M.nparam);
    M.d_v = (float*)dalloc(ctx, sizeof(float) * M.nparam);
    M.d_g = (float*)dalloc(ctx, sizeof(float) * M.nparam);
    MWB_CUDA(cudaMemcpyAsync(M.d_p, p.data(), sizeof(float) * M.nparam, cudaMemcpyHostToDevice, s));
    MWB_CUDA(cudaMemsetAsync(M.d_m, 0, sizeof(float) * M.nparam, s));
    MWB_CUDA(cudaMemsetAsync(M.d_v, 0, sizeof(float) * M.nparam, s));
    MWB_CUDA(cudaStreamSynchronize(s));
}

// forward over N rows of X; keeps the activations of every layer in acts (for backward)
void mlp_forward(Mlp& M, const float* d_X, int N, std::vector<float*>& acts, cudaStream_t s) {
    const int L = (int)M.dims.size() - 1;
    acts.assign(L + 1, nullptr);
    acts[0] = const_cast<float*>(d_X);
    for (int l = 0; l < L; ++l) {
        acts[l + 1] = (float*)dalloc(M.ctx, sizeof(float) * (size_t)N * M.dims[l + 1]);
        dim3 blk(16, 16), grd((N + 15) / 16, (M.dims[l + 1] + 15) / 16);
        k_lin_fwd<<<grd, blk, 0, s>>>(acts[l], M.d_p + M.woff[l], M.d_p + M.boff[l], acts[l + 1], N, M.dims[l],
                                      M.dims[l + 1], l + 1 < L ? 1 : 0);
    }
    MWB_CUDA(cudaGetLastError());
}

// gradient of the weighted BCE loss into d_g; returns the loss
double mlp_backward(Mlp& M, std::vector<float*>& acts, const float* d_y, const float* d_w, int N, cudaStream_t s) {
    const int L = (int)M.dims.size() - 1;
    Ctx* ctx = M.ctx;
    float* dz = (float*)dalloc(ctx, sizeof(float) * N);
    const int nb = 120;
    float* d_lp = (float*)dalloc(ctx, sizeof(float) * nb);
    k_bce<<<nb, 256, 0, s>>>(acts[L], d_y, d_w, N, dz, d_lp);
    float* dcur = dz;
    for (int l = L - 1; l >= 0; --l) {
        dim3 blk(16, 16);
        k_lin_bwd_w<<<dim3((M.dims[l] + 15) / 16, (M.dims[l + 1] + 15) / 16), blk, 0, s>>>(
            dcur, acts[l], M.d_g + M.woff[l], M.d_g + M.boff[l], N, M.dims[l], M.dims[l + 1]);
        if (l > 0) {
            float* dprev = (float*)dalloc(ctx, sizeof(float) * (size_t)N * M.dims[l]);
            k_lin_bwd_x<<<dim3((N + 15) / 16, (M.dims[l] + 15) / 16), blk, 0, s>>>(dcur, M.d_p + M.woff[l], dprev, N,
                                                                                     M.dims[l], M.dims[l + 1]);
            k_relu_mask<<<256, 256, 0, s>>>(dprev, acts[l], (size_t)N * M.dims[l]);
            if (dcur != dz) dfree(ctx, dcur);
            dcur = dprev;
        }
    }
    MWB_CUDA(cudaGetLastError());
    if (dcur != dz) dfree(ctx, dcur);
    std::vector<float> lp(nb);
    MWB_CUDA(cudaMemcpyAsync(lp.data(), d_lp, sizeof(float) * nb, cudaMemcpyDeviceToHost, s));
    MWB_CUDA(cudaStreamSynchronize(s));
    dfree(ctx, dz);
    dfree(ctx, d_lp);
    double loss = 0.0;
    for (float v : lp) loss += v;
    return loss / N;
}

void free_acts(Mlp& M, std::vector<float*>& acts) {
    for (size_t l = 1; l < acts.size(); ++l) dfree(M.ctx, acts[l]);
    acts.clear();
}

// logits of N feature rows already on the device
std::vector<float> mlp_logits(Mlp& M, const float* d_X, int N, cudaStream_t s) {
    std::vector<float*> acts;
    mlp_forward(M, d_X, N, acts, s);
    std::vector<float> z(N);
    readback(M.ctx, s, {{z.data(), acts.back(), sizeof(float) * N}});
    free_acts(M, acts);
    return z;
}

// ---------------------------------------------------------------------------------------------
// features of a node list of several trees
// ---------------------------------------------------------------------------------------------
float* features(Ctx* ctx, std::vector<FeatCtx>& fc, const std::vector<int2>& items, cudaStream_t s) {
    const int n = (int)items.size();
    float* d_F = (float*)dalloc(ctx, sizeof(float) * (size_t)std::max(1, n) * kNF);
    if (n == 0) return d_F;
    std::vector<FeatTree> ft(fc.size());
    for (size_t t = 0; t < fc.size(); ++t) {
        FeatCtx& c = fc[t];
        const Mra& m = *c.out->mra;
        FeatTree& f = ft[t];
        f.okey = c.out->key;
        f.ikey = c.inp->key;
        f.inorm2 = c.inp->norm2;
        f.iwnorm2 = c.inp->wnorm2;
        f.hkey = c.inp->hkey;
        f.hval = c.inp->hval;
        f.hcap = c.inp->hcap;
        f.owind2 = c.out->wnorm2;
        f.ohkey = c.out->hkey;
        f.ohval = c.out->hval;
        f.ohcap = c.out->hcap;
        f.n0 = m.n0;
        for (int q = 0; q < 3; ++q) f.boxes[q] = m.boxes[q];
        f.thr0 = c.prec * c.g0;
        f.mu = c.op->mu;
        f.prec = c.prec;
    }
    FeatTree* d_ft = (FeatTree*)dalloc(ctx, sizeof(FeatTree) * ft.size());
    int2* d_items = (int2*)dalloc(ctx, sizeof(int2) * n);
    upload_bytes(ctx, s, d_ft, ft.data(), sizeof(FeatTree) * ft.size());  // staged: ft / items may go
    upload_bytes(ctx, s, d_items, items.data(), sizeof(int2) * n);
    k_features<<<(unsigned)(((size_t)n * 32 + 255) / 256), 256, 0, s>>>(d_items, n, d_ft, d_F);  // a warp per node
    MWB_CUDA(cudaGetLastError());
    if (s != ctx->stream) MWB_CUDA(cudaStreamSynchronize(s));  // pageable copies: ft / items leave scope
    dfree(ctx, d_ft);
    dfree(ctx, d_items);
    return d_F;
}

// ---------------------------------------------------------------------------------------------
// training set collection from a plain apply (labels: the node was split)
// ---------------------------------------------------------------------------------------------
void mlp_append(Mlp& M, const float* d_F, const std::vector<float>& y, cudaStream_t s) {
    const int n = (int)y.size();
    if (M.n_data + n > M.cap_data) {
        int ncap = std::max(M.n_data + n, 2 * M.cap_data + 1024);
        float* X = (float*)dalloc(M.ctx, sizeof(float) * (size_t)ncap * kNF);
        float* Y = (float*)dalloc(M.ctx, sizeof(float) * ncap);
        if (M.n_data) {
            MWB_CUDA(cudaMemcpyAsync(X, M.d_X, sizeof(float) * (size_t)M.n_data * kNF, cudaMemcpyDeviceToDevice, s));
            MWB_CUDA(cudaMemcpyAsync(Y, M.d_y, sizeof(float) * M.n_data, cudaMemcpyDeviceToDevice, s));
        }
        dfree(M.ctx, M.d_X);
        dfree(M.ctx, M.d_y);
        M.d_X = X;
        M.d_y = Y;
        M.cap_data = ncap;
    }
    MWB_CUDA(cudaMemcpyAsync(M.d_X + (size_t)M.n_data * kNF, d_F, sizeof(float) * (size_t)n * kNF,
                             cudaMemcpyDeviceToDevice, s));
    MWB_CUDA(cudaMemcpyAsync(M.d_y + M.n_data, y.data(), sizeof(float) * n, cudaMemcpyHostToDevice, s));
    MWB_CUDA(cudaStreamSynchronize(s));
    M.n_data += n;
}

// ---------------------------------------------------------------------------------------------
// tree surgery: keep a subset of nodes and rebuild in (depth, Morton) order
// ---------------------------------------------------------------------------------------------
__global__ void k_gather_nodes(const double* __restrict__ coef, const double* __restrict__ n2,
                               const double* __restrict__ w2, const uint64_t* __restrict__ key,
                               const int* __restrict__ perm, int n, size_t bs, double* ncoef, double* nn2, double* nw2,
                               uint64_t* nkey) {
    const int i = blockIdx.x;
    if (i >= n) return;
    const int o = perm[i];
    for (size_t e = threadIdx.x; e < bs; e += blockDim.x) ncoef[(size_t)i * bs + e] = coef[(size_t)o * bs + e];
    if (threadIdx.x == 0) {
        nn2[i] = n2[o];
        nw2[i] = w2[o];
        nkey[i] = key[o];
    }
}

// Rebuild each tree keeping the nodes whose flag is set (every kept node's parent kept, siblings kept
// together), reordered by key so that parents precede children; keys[i] are the trees' current
// node keys (host copies).  All trees are rebuilt with one synchronisation.
void trees_rebuild(const std::vector<Tree*>& ts, const std::vector<std::vector<char>>& keeps,
                   const std::vector<std::vector<uint64_t>>& keys) {
    if (ts.empty()) return;
    Ctx* ctx = ts[0]->mra->ctx;
    cudaStream_t s = ctx->stream;
    const size_t BS = ts[0]->mra->bsize();
    struct Host {
        std::vector<int> perm, parent, child0;
        int* d_perm;
        double *ncoef, *nn2, *nw2;
        uint64_t* nkey;
    };
    std::vector<Host> H(ts.size());
    for (size_t q = 0; q < ts.size(); ++q) {
        Tree& t = *ts[q];
        const std::vector<uint64_t>& key = keys[q];
        Host& h = H[q];
        for (int i = 0; i < t.n; ++i)
            if (keeps[q][i]) h.perm.push_back(i);
        std::sort(h.perm.begin(), h.perm.end(), [&](int a, int b) { return key[a] < key[b]; });
        const int nn = (int)h.perm.size();
        std::unordered_map<uint64_t, int> pos;
        pos.reserve(2 * nn);
        for (int i = 0; i < nn; ++i) pos[key[h.perm[i]]] = i;
        h.parent.assign(nn, -1);
        h.child0.assign(nn, -1);
        int maxd = 0;
        for (int i = 0; i < nn; ++i) {
            const uint64_t k = key[h.perm[i]];
            const int d = (int)(k >> 59);
            maxd = std::max(maxd, d);
            long long tr[3];
            host_key_trans(k, tr);
            if (d > 0) h.parent[i] = pos.at(host_make_key(d - 1, tr[0] >> 1, tr[1] >> 1, tr[2] >> 1));
            auto it = pos.find(host_make_key(d + 1, 2 * tr[0], 2 * tr[1], 2 * tr[2]));
            if (it != pos.end()) h.child0[i] = it->second;
        }
        std::vector<int> lb(maxd + 2, 0);
        for (int i = 0; i < nn; ++i) lb[(key[h.perm[i]] >> 59) + 1]++;
        for (size_t d = 1; d < lb.size(); ++d) lb[d] += lb[d - 1];
        h.d_perm = (int*)dalloc(ctx, sizeof(int) * std::max(1, nn));
        h.ncoef = (double*)dalloc(ctx, sizeof(double) * BS * std::max(1, nn));
        h.nn2 = (double*)dalloc(ctx, sizeof(double) * std::max(1, nn));
        h.nw2 = (double*)dalloc(ctx, sizeof(double) * std::max(1, nn));
        h.nkey = (uint64_t*)dalloc(ctx, sizeof(uint64_t) * std::max(1, nn));
        MWB_CUDA(cudaMemcpyAsync(h.d_perm, h.perm.data(), sizeof(int) * nn, cudaMemcpyHostToDevice, s));
        k_gather_nodes<<<nn, 256, 0, s>>>(t.coef, t.norm2, t.wnorm2, t.key, h.d_perm, nn, BS, h.ncoef, h.nn2, h.nw2,
                                          h.nkey);
        MWB_CUDA(cudaGetLastError());
        MWB_CUDA(cudaMemcpyAsync(t.coef, h.ncoef, sizeof(double) * BS * nn, cudaMemcpyDeviceToDevice, s));
        MWB_CUDA(cudaMemcpyAsync(t.norm2, h.nn2, sizeof(double) * nn, cudaMemcpyDeviceToDevice, s));
        MWB_CUDA(cudaMemcpyAsync(t.wnorm2, h.nw2, sizeof(double) * nn, cudaMemcpyDeviceToDevice, s));
        MWB_CUDA(cudaMemcpyAsync(t.key, h.nkey, sizeof(uint64_t) * nn, cudaMemcpyDeviceToDevice, s));
        MWB_CUDA(cudaMemcpyAsync(t.parent, h.parent.data(), sizeof(int) * nn, cudaMemcpyHostToDevice, s));
        MWB_CUDA(cudaMemcpyAsync(t.child0, h.child0.data(), sizeof(int) * nn, cudaMemcpyHostToDevice, s));
        t.n = nn;
        t.level_begin = lb;
        launch_hash_reset(t, s);
        launch_hash_insert(t, 0, nn, s);
    }
    MWB_CUDA(cudaStreamSynchronize(s));
    for (Host& h : H)
        for (void* p : {(void*)h.d_perm, (void*)h.ncoef, (void*)h.nn2, (void*)h.nw2, (void*)h.nkey}) dfree(ctx, p);
}

// class-balanced weights for the current training set
static std::vector<float> balance_weights(const std::vector<float>& y) {
    double npos = 0.0;
    for (float v : y) npos += v;
    const double n = (double)y.size(), nneg = n - npos;
    const float wp = npos > 0 ? (float)(n / (2.0 * npos)) : 0.0f, wn = nneg > 0 ? (float)(n / (2.0 * nneg)) : 0.0f;
    std::vector<float> w(y.size());
    for (size_t i = 0; i < y.size(); ++i) w[i] = y[i] > 0.5f ? wp : wn;
    return w;
}

double mlp_train(Mlp& M, int epochs, int batch, float lr, unsigned seed) {
    Ctx* ctx = M.ctx;
    cudaStream_t s = ctx->stream;
    const int N = M.n_data;
    if (N == 0) throw Error(-3, "empty training set");
    std::vector<float> y(N);
    MWB_CUDA(cudaMemcpyAsync(y.data(), M.d_y, sizeof(float) * N, cudaMemcpyDeviceToHost, s));
    MWB_CUDA(cudaStreamSynchronize(s));
    const std::vector<float> w = balance_weights(y);
    float* d_w = (float*)dalloc(ctx, sizeof(float) * N);
    MWB_CUDA(cudaMemcpyAsync(d_w, w.data(), sizeof(float) * N, cudaMemcpyHostToDevice, s));
    batch = std::max(1, std::min(batch, N));
    float* d_bx = (float*)dalloc(ctx, sizeof(float) * (size_t)batch * kNF);
    float* d_by = (float*)dalloc(ctx, sizeof(float) * batch);
    float* d_bw = (float*)dalloc(ctx, sizeof(float) * batch);
    int* d_idx = (int*)dalloc(ctx, sizeof(int) * batch);
    std::vector<int> perm(N);
    std::iota(perm.begin(), perm.end(), 0);
    std::mt19937 rng(seed);
    double last = 0.0;
    const float b1 = 0.9f, b2 = 0.999f;
    for (int ep = 0; ep < epochs; ++ep) {
        std::shuffle(perm.begin(), perm.end(), rng);
        double tot = 0.0;
        int nb = 0;
        for (int b0 = 0; b0 + batch <= N || (b0 < N && nb == 0); b0 += batch) {
            const int bn = std::min(batch, N - b0);
            MWB_CUDA(cudaMemcpyAsync(d_idx, perm.data() + b0, sizeof(int) * bn, cudaMemcpyHostToDevice, s));
            k_gather_rows<<<bn, 64, 0, s>>>(M.d_X, d_idx, bn, kNF, d_bx);
            k_gather_rows<<<bn, 32, 0, s>>>(M.d_y, d_idx, bn, 1, d_by);
            k_gather_rows<<<bn, 32, 0, s>>>(d_w, d_idx, bn, 1, d_bw);
            std::vector<float*> acts;
            mlp_forward(M, d_bx, bn, acts, s);
            tot += mlp_backward(M, acts, d_by, d_bw, bn, s);
            free_acts(M, acts);
            ++M.adam_t;
            const float c1 = 1.0f - std::pow(b1, (float)M.adam_t), c2 = 1.0f - std::pow(b2, (float)M.adam_t);
            k_adam<<<((int)M.nparam + 255) / 256, 256, 0, s>>>(M.d_p, M.d_g, M.d_m, M.d_v, (int)M.nparam, lr, b1, b2,
                                                               1e-8f, c1, c2);
            MWB_CUDA(cudaGetLastError());
            ++nb;
        }
        last = tot / std::max(1, nb);
    }
    MWB_CUDA(cudaStreamSynchronize(s));
    for (void* q : {(void*)d_w, (void*)d_bx, (void*)d_by, (void*)d_bw, (void*)d_idx}) dfree(ctx, q);
    return last;
}

}  // namespace mwb

namespace mwb {

// ---------------------------------------------------------------------------------------------
// exact criterion and rebuild on the device
// ---------------------------------------------------------------------------------------------
namespace {
constexpr int kMaxLevels = 64;

struct VTree {
    const uint64_t* key;
    const int* parent;
    const int* child0;
    const double* wnorm2;
    int n;
    long long off;
};

// one thread per node of tree blockIdx.y: keep = all strict ancestors split; a kept node that splits
// without children is appended to the miss list
__global__ void k_verify(const VTree* __restrict__ ts, const double* __restrict__ thr, int depth_limit,
                         unsigned char* keep, int* nmiss, Miss* miss, int cap) {
    const VTree T = ts[blockIdx.y];
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= T.n) return;
    const double* th = thr + (size_t)blockIdx.y * kMaxLevels;
    auto splits = [&](int p) {
        const int d = key_depth(T.key[p]);
        return d < depth_limit && sqrt(T.wnorm2[p]) > th[d];
    };
    unsigned char k = 1;
    for (int p = T.parent[q]; p >= 0; p = T.parent[p])
        if (!splits(p)) {
            k = 0;
            break;
        }
    keep[T.off + q] = k;
    if (k && T.child0[q] < 0 && splits(q)) {
        const int w = atomicAdd(nmiss, 1);
        if (w < cap) miss[w] = Miss{(int)blockIdx.y, q, T.key[q]};
    }
}

struct RTree {  // old arrays, new arrays and hash index of one tree being rebuilt
    const uint64_t* okey;
    const double* ocoef;
    const double* on2;
    const double* ow2;
    uint64_t* nkey;
    double* ncoef;
    double* nn2;
    double* nw2;
    int* nparent;
    int* nchild0;
    const uint64_t* hkey;
    const int* hval;
    uint32_t hcap;
    long long off;   // first global index of the tree's old nodes
    long long noff;  // first position of the tree's kept nodes in the sorted list
    int nn;
    int cap;  // capacity of the new arrays
};

__global__ void k_gather_keys(const uint64_t* __restrict__ k, const long long* __restrict__ g, int n, uint64_t* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = k[g[i]];
}

// tree of each kept node (largest tree whose first global index is <= g[i]); kept nodes per tree
__global__ void k_tree_of(const long long* __restrict__ g, int n, const long long* __restrict__ offs, int nt,
                          unsigned* tid, int* cnt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int lo = 0, hi = nt - 1;  // last tree whose offset <= g[i]
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (offs[mid] <= g[i]) lo = mid;
        else hi = mid - 1;
    }
    tid[i] = (unsigned)lo;
    atomicAdd(&cnt[lo], 1);
}

// block j: kept node j of the sorted list (tree tid[j]) -> its new position
__global__ void k_rebuild_gather(const long long* __restrict__ g, const unsigned* __restrict__ tid, int n,
                                 const RTree* __restrict__ rt, size_t bs) {
    const int j = blockIdx.x;
    if (j >= n) return;
    const RTree& R = rt[tid[j]];
    const long long o = g[j] - R.off;
    const long long d = j - R.noff;
    const double* src = R.ocoef + (size_t)o * bs;
    double* dst = R.ncoef + (size_t)d * bs;
    for (size_t e = threadIdx.x; e < bs; e += blockDim.x) dst[e] = src[e];
    if (threadIdx.x == 0) {
        R.nkey[d] = R.okey[o];
        R.nn2[d] = R.on2[o];
        R.nw2[d] = R.ow2[o];
    }
}

// parent and first child of every new node from the rebuilt hash index; level starts per tree
__global__ void k_rebuild_links(const unsigned* __restrict__ tid, int n, const RTree* __restrict__ rt, int* lb) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const unsigned t = tid[j];
    const RTree& R = rt[t];
    const int d = (int)(j - R.noff);
    const uint64_t k = R.nkey[d];
    const int dep = key_depth(k);
    long long tr[3];
    key_trans(k, tr);
    R.nparent[d] = dep > 0 ? hlookup(R.hkey, R.hval, R.hcap, make_key(dep - 1, tr[0] >> 1, tr[1] >> 1, tr[2] >> 1)) : -1;
    R.nchild0[d] = hlookup(R.hkey, R.hval, R.hcap, make_key(dep + 1, 2 * tr[0], 2 * tr[1], 2 * tr[2]));
    if (d == 0 || key_depth(R.nkey[d - 1]) != dep) lb[(size_t)t * (kMaxLevels + 1) + dep] = d;
}
}  // namespace

std::vector<Miss> verify_trees(const std::vector<Tree*>& ts, const std::vector<std::vector<double>>& thr,
                               int depth_limit, unsigned char* d_keep, cudaStream_t s) {
    const int nt = (int)ts.size();
    if (nt == 0) return {};
    Ctx* ctx = ts[0]->mra->ctx;
    std::vector<VTree> vt(nt);
    std::vector<double> th((size_t)nt * kMaxLevels, INFINITY);
    long long off = 0;
    int maxn = 0;
    for (int i = 0; i < nt; ++i) {
        const Tree& t = *ts[i];
        vt[i] = VTree{t.key, t.parent, t.child0, t.wnorm2, t.n, off};
        off += t.n;
        maxn = std::max(maxn, t.n);
        for (int d = 0; d < kMaxLevels && d < (int)thr[i].size(); ++d) th[(size_t)i * kMaxLevels + d] = thr[i][d];
    }
    if (depth_limit > kMaxLevels) throw Error(-3, "depth limit beyond the verification table");
    VTree* d_vt = (VTree*)dalloc(ctx, sizeof(VTree) * nt);
    double* d_th = (double*)dalloc(ctx, sizeof(double) * th.size());
    int cap = 4096;
    std::vector<Miss> out;
    for (;;) {
        int* d_n = (int*)dalloc(ctx, sizeof(int));
        Miss* d_m = (Miss*)dalloc(ctx, sizeof(Miss) * cap);
        upload_bytes(ctx, s, d_vt, vt.data(), sizeof(VTree) * nt);
        upload_bytes(ctx, s, d_th, th.data(), sizeof(double) * th.size());
        MWB_CUDA(cudaMemsetAsync(d_n, 0, sizeof(int), s));
        if (maxn > 0) {
            k_verify<<<dim3((maxn + 255) / 256, nt), 256, 0, s>>>(d_vt, d_th, depth_limit, d_keep, d_n, d_m, cap);
            MWB_CUDA(cudaGetLastError());
        }
        int nm = 0;
        readback(ctx, s, {{&nm, d_n, sizeof(int)}});
        if (nm <= cap) {
            out.resize(nm);
            if (nm > 0) readback(ctx, s, {{out.data(), d_m, sizeof(Miss) * nm}});
            dfree(ctx, d_n);
            dfree(ctx, d_m);
            break;
        }
        dfree(ctx, d_n);
        dfree(ctx, d_m);
        cap = nm;  // the list did not fit: once more with room for all
    }
    dfree(ctx, d_vt);
    dfree(ctx, d_th);
    return out;
}

long long trees_rebuild_device(const std::vector<Tree*>& ts, const unsigned char* d_keep, cudaStream_t s) {
    const int nt = (int)ts.size();
    if (nt == 0) return 0;
    Ctx* ctx = ts[0]->mra->ctx;
    const size_t BS = ts[0]->mra->bsize();
    std::vector<long long> offs(nt + 1, 0);
    for (int i = 0; i < nt; ++i) offs[i + 1] = offs[i] + ts[i]->n;
    const long long total = offs[nt];
    if (total <= 0) return 0;
    if (total > (1LL << 31) - 1) throw Error(-4, "too many nodes to rebuild at once");
    const int N = (int)total;
    // keys of all nodes, concatenated
    uint64_t* d_k = (uint64_t*)dalloc(ctx, sizeof(uint64_t) * N);
    for (int i = 0; i < nt; ++i)
        if (ts[i]->n > 0)
            device_copy(ctx, d_k + offs[i], ts[i]->key, sizeof(uint64_t) * ts[i]->n);  // on s (= the context's stream)
    // kept global indices, ascending (grouped by tree)
    long long* d_g = (long long*)dalloc(ctx, sizeof(long long) * N);
    int* d_nsel = (int*)dalloc(ctx, sizeof(int));
    {
        thrust::counting_iterator<long long> cnt(0);
        size_t tmp = 0;
        MWB_CUDA(cub::DeviceSelect::Flagged(nullptr, tmp, cnt, d_keep, d_g, d_nsel, N, s));
        void* d_tmp = dalloc(ctx, std::max<size_t>(tmp, 1));
        MWB_CUDA(cub::DeviceSelect::Flagged(d_tmp, tmp, cnt, d_keep, d_g, d_nsel, N, s));
        dfree(ctx, d_tmp);
    }
    int n = 0;
    readback(ctx, s, {{&n, d_nsel, sizeof(int)}});
    // sort the kept nodes by key, then stably by tree: grouped by tree, key order inside a tree
    uint64_t* d_kk = (uint64_t*)dalloc(ctx, sizeof(uint64_t) * std::max(1, n));
    uint64_t* d_kk2 = (uint64_t*)dalloc(ctx, sizeof(uint64_t) * std::max(1, n));
    long long* d_g2 = (long long*)dalloc(ctx, sizeof(long long) * std::max(1, n));
    unsigned* d_tid = (unsigned*)dalloc(ctx, sizeof(unsigned) * std::max(1, n));
    unsigned* d_tid2 = (unsigned*)dalloc(ctx, sizeof(unsigned) * std::max(1, n));
    long long* d_offs = (long long*)dalloc(ctx, sizeof(long long) * (nt + 1));
    int* d_cnt = (int*)dalloc(ctx, sizeof(int) * nt);
    upload_bytes(ctx, s, d_offs, offs.data(), sizeof(long long) * (nt + 1));
    MWB_CUDA(cudaMemsetAsync(d_cnt, 0, sizeof(int) * nt, s));
    k_gather_keys<<<(n + 255) / 256, 256, 0, s>>>(d_k, d_g, n, d_kk);
    {
        size_t tmp = 0;
        MWB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, d_kk, d_kk2, d_g, d_g2, n, 0, 64, s));
        void* d_tmp = dalloc(ctx, std::max<size_t>(tmp, 1));
        MWB_CUDA(cub::DeviceRadixSort::SortPairs(d_tmp, tmp, d_kk, d_kk2, d_g, d_g2, n, 0, 64, s));
        dfree(ctx, d_tmp);
    }
    k_tree_of<<<(n + 255) / 256, 256, 0, s>>>(d_g2, n, d_offs, nt, d_tid, d_cnt);
    {
        int bits = 1;
        while ((1 << bits) < nt) ++bits;
        size_t tmp = 0;
        MWB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, d_tid, d_tid2, d_g2, d_g, n, 0, bits, s));
        void* d_tmp = dalloc(ctx, std::max<size_t>(tmp, 1));
        MWB_CUDA(cub::DeviceRadixSort::SortPairs(d_tmp, tmp, d_tid, d_tid2, d_g2, d_g, n, 0, bits, s));
        dfree(ctx, d_tmp);
    }
    MWB_CUDA(cudaGetLastError());
    std::vector<int> cnt(nt);
    readback(ctx, s, {{cnt.data(), d_cnt, sizeof(int) * nt}});
    // new arrays, gather, swap
    std::vector<RTree> rt(nt);
    long long noff = 0;
    for (int i = 0; i < nt; ++i) {
        Tree& t = *ts[i];
        const int nn = cnt[i];
        RTree& R = rt[i];
        R.okey = t.key;
        R.ocoef = t.coef;
        R.on2 = t.norm2;
        R.ow2 = t.wnorm2;
        // room beyond the kept nodes: the next apply into this tree (proposals overshoot) grows it in place
        const int capn = nn + nn / 4 + 64;
        R.cap = capn;
        R.nkey = (uint64_t*)dalloc(ctx, sizeof(uint64_t) * capn);
        R.ncoef = (double*)dalloc(ctx, sizeof(double) * BS * capn);
        R.nn2 = (double*)dalloc(ctx, sizeof(double) * capn);
        R.nw2 = (double*)dalloc(ctx, sizeof(double) * capn);
        R.nparent = (int*)dalloc(ctx, sizeof(int) * capn);
        R.nchild0 = (int*)dalloc(ctx, sizeof(int) * capn);
        R.hkey = t.hkey;
        R.hval = t.hval;
        R.hcap = t.hcap;
        R.off = offs[i];
        R.noff = noff;
        R.nn = nn;
        noff += nn;
    }
    RTree* d_rt = (RTree*)dalloc(ctx, sizeof(RTree) * nt);
    upload_bytes(ctx, s, d_rt, rt.data(), sizeof(RTree) * nt);
    if (n > 0) k_rebuild_gather<<<n, 256, 0, s>>>(d_g, d_tid2, n, d_rt, BS);
    MWB_CUDA(cudaGetLastError());
    for (int i = 0; i < nt; ++i) {
        Tree& t = *ts[i];
        RTree& R = rt[i];
        dfree(ctx, t.key);
        dfree(ctx, t.coef);
        dfree(ctx, t.norm2);
        dfree(ctx, t.wnorm2);
        dfree(ctx, t.parent);
        dfree(ctx, t.child0);
        t.key = R.nkey;
        t.coef = R.ncoef;
        t.norm2 = R.nn2;
        t.wnorm2 = R.nw2;
        t.parent = R.nparent;
        t.child0 = R.nchild0;
        t.n = R.nn;
        t.cap = R.cap;
        if (s != ctx->stream) {
            launch_hash_reset(t, s);
            launch_hash_insert(t, 0, t.n, s);
        }
    }
    if (s == ctx->stream) trees_rehash(ts);  // all the rebuilt indices in two launches
    // links and level starts from the rebuilt hash indices
    int* d_lb = (int*)dalloc(ctx, sizeof(int) * (size_t)nt * (kMaxLevels + 1));
    MWB_CUDA(cudaMemsetAsync(d_lb, 0xff, sizeof(int) * (size_t)nt * (kMaxLevels + 1), s));
    if (n > 0) k_rebuild_links<<<(n + 255) / 256, 256, 0, s>>>(d_tid2, n, d_rt, d_lb);
    MWB_CUDA(cudaGetLastError());
    std::vector<int> lb((size_t)nt * (kMaxLevels + 1));
    readback(ctx, s, {{lb.data(), d_lb, sizeof(int) * lb.size()}});
    for (int i = 0; i < nt; ++i) {
        Tree& t = *ts[i];
        const int* L = lb.data() + (size_t)i * (kMaxLevels + 1);
        int maxd = 0;
        for (int d = 0; d < kMaxLevels; ++d)
            if (L[d] >= 0) maxd = d;
        t.level_begin.assign(maxd + 2, 0);
        for (int d = 0; d <= maxd; ++d) {
            if (L[d] < 0) throw Error(-3, "rebuilt tree has an empty level");
            t.level_begin[d] = L[d];
        }
        t.level_begin[maxd + 1] = t.n;
    }
    for (void* p : std::initializer_list<void*>{d_k, d_g, d_nsel, d_kk, d_kk2, d_g2, d_tid, d_tid2, d_offs, d_cnt, d_rt,
                                                d_lb})
        dfree(ctx, p);
    return total - n;
}

}  // namespace mwb
