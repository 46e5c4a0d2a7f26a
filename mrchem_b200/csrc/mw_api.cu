// mw_api.cu -- host driver behind the C-ABI (include/mwb200.h): contexts, worlds, device trees,
// operator tables, and the adaptive projection / apply loops that issue the sm_100a kernels.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>
#include <string>
#include <tuple>
#include <unordered_map>

#include "../../include/mwb200.h"
#include "mw_kernels.cuh"
#include "mw_slice.hpp"
#include "mw_learned.cuh"

namespace mwb {


static thread_local std::string g_err;

// lets other translation units of the C-ABI report an error through mw_last_error()
void set_last_error(const std::string& msg) { g_err = msg; }

void* dalloc(Ctx* ctx, size_t bytes) {
    void* p = nullptr;
    if (bytes == 0) bytes = 16;
    MWB_CUDA(cudaMallocAsync(&p, bytes, ctx->stream));
    return p;
}
void dfree(Ctx* ctx, void* p) {
    if (p) cudaFreeAsync(p, ctx->stream);
}
// copies of up to 8 byte ranges in one launch (grid-stride, 16- or 4-byte words where both ends allow)
struct CopyList {
    const unsigned char* src[8];
    unsigned char* dst[8];
    unsigned long long n[8];
    int count;
};
__global__ void k_copy_list(CopyList L) {
    const size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x, nth = (size_t)gridDim.x * blockDim.x;
    for (int r = 0; r < L.count; ++r) {
        const unsigned char* src = L.src[r];
        unsigned char* dst = L.dst[r];
        const size_t n = L.n[r];
        const uintptr_t al = reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst);
        size_t done = 0;
        if ((al & 15) == 0) {
            const size_t nw = n >> 4;
            for (size_t i = tid; i < nw; i += nth) reinterpret_cast<uint4*>(dst)[i] = reinterpret_cast<const uint4*>(src)[i];
            done = nw << 4;
        } else if ((al & 3) == 0) {
            const size_t nw = n >> 2;
            for (size_t i = tid; i < nw; i += nth)
                reinterpret_cast<uint32_t*>(dst)[i] = reinterpret_cast<const uint32_t*>(src)[i];
            done = nw << 2;
        }
        for (size_t i = done + tid; i < n; i += nth) dst[i] = src[i];
    }
}
static void launch_copies(Ctx* ctx, const CopyList& L) {
    size_t mx = 0;
    for (int r = 0; r < L.count; ++r) mx = std::max<size_t>(mx, L.n[r]);
    const int blocks = (int)std::max<size_t>(1, std::min<size_t>(512, (mx / 16 + 255) / 256));
    k_copy_list<<<blocks, 256, 0, ctx->stream>>>(L);
    MWB_CUDA(cudaGetLastError());
    ctx->launches += 1;
}

void upload_bytes(Ctx* ctx, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return;
    constexpr size_t kArena = 32u << 20;
    if (!ctx->pin && bytes <= kArena / 4) {
        MWB_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&ctx->pin), kArena, cudaHostAllocMapped));
        MWB_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void**>(&ctx->pin_dev), ctx->pin, 0));
        MWB_CUDA(cudaEventCreateWithFlags(&ctx->pin_ev, cudaEventDisableTiming));
        ctx->pin_cap = kArena;
        ctx->pin_off = 0;
    }
    if (!ctx->pin || bytes > ctx->pin_cap / 4) {  // large: pageable copy
        MWB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
        return;
    }
    if (ctx->pin_off + bytes > ctx->pin_cap) {  // wrap: every earlier copy from the arena has completed
        if (ctx->pin_pending) MWB_CUDA(cudaEventSynchronize(ctx->pin_ev));
        ctx->pin_off = 0;
    }
    std::memcpy(ctx->pin + ctx->pin_off, src, bytes);
    CopyList L{};
    L.src[0] = reinterpret_cast<const unsigned char*>(ctx->pin_dev + ctx->pin_off);
    L.dst[0] = reinterpret_cast<unsigned char*>(dst);
    L.n[0] = bytes;
    L.count = 1;
    launch_copies(ctx, L);
    MWB_CUDA(cudaEventRecord(ctx->pin_ev, ctx->stream));
    ctx->pin_pending = true;
    ctx->pin_off += (bytes + 255) & ~(size_t)255;
}

void readback(Ctx* ctx, std::initializer_list<ReadReq> reqs) {
    constexpr size_t kBox = 4u << 20;
    if (!ctx->mbox) {
        MWB_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&ctx->mbox), kBox, cudaHostAllocMapped));
        MWB_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void**>(&ctx->mbox_dev), ctx->mbox, 0));
        ctx->mbox_cap = kBox;
    }
    if (reqs.size() > 8) throw Error(MW_ERR_ARG, "readback: at most 8 ranges");
    CopyList L{};
    long long at[8];  // mailbox offset of each request, -1: empty or through the copy engine
    size_t used = 0;
    int i = 0;
    for (const ReadReq& r : reqs) {
        at[i] = -1;
        const size_t o = (used + 15) & ~(size_t)15;
        if (r.bytes > 0 && o + r.bytes <= ctx->mbox_cap) {
            at[i] = (long long)o;
            L.src[L.count] = reinterpret_cast<const unsigned char*>(r.src);
            L.dst[L.count] = reinterpret_cast<unsigned char*>(ctx->mbox_dev + o);
            L.n[L.count] = r.bytes;
            ++L.count;
            used = o + r.bytes;
        }
        ++i;
    }
    if (L.count > 0) launch_copies(ctx, L);
    i = 0;
    for (const ReadReq& r : reqs) {  // what does not fit the mailbox (pageable: completes in the call)
        if (r.bytes > 0 && at[i] < 0) MWB_CUDA(cudaMemcpyAsync(r.dst, r.src, r.bytes, cudaMemcpyDeviceToHost, ctx->stream));
        ++i;
    }
    MWB_CUDA(cudaStreamSynchronize(ctx->stream));
    i = 0;
    for (const ReadReq& r : reqs) {
        if (at[i] >= 0) std::memcpy(r.dst, ctx->mbox + at[i], r.bytes);
        ++i;
    }
}

void upload_bytes(Ctx* ctx, cudaStream_t s, void* dst, const void* src, size_t bytes) {
    if (s == ctx->stream) upload_bytes(ctx, dst, src, bytes);
    else if (bytes > 0) MWB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
}
void device_copy(Ctx* ctx, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return;
    CopyList L{};
    L.src[0] = reinterpret_cast<const unsigned char*>(src);
    L.dst[0] = reinterpret_cast<unsigned char*>(dst);
    L.n[0] = bytes;
    L.count = 1;
    launch_copies(ctx, L);
}
void readback(Ctx* ctx, cudaStream_t s, std::initializer_list<ReadReq> reqs) {
    if (s == ctx->stream) {
        readback(ctx, reqs);
        return;
    }
    for (const ReadReq& r : reqs)
        if (r.bytes > 0) MWB_CUDA(cudaMemcpyAsync(r.dst, r.src, r.bytes, cudaMemcpyDeviceToHost, s));
    MWB_CUDA(cudaStreamSynchronize(s));
}

// ---------------------------------------------------------------------------------------------
// screening constants of the apply (same values as the CPU oracle)
// ---------------------------------------------------------------------------------------------
constexpr double kScreen = 0.1;  // skip a contribution below kScreen x the output split threshold
inline double split_threshold(double prec, double ref, int depth) { return prec * ref * std::pow(2.0, -0.5 * depth); }

// ---------------------------------------------------------------------------------------------
// trees
// ---------------------------------------------------------------------------------------------

Tree::~Tree() {
    if (!mra) return;
    Ctx* c = mra->ctx;
    cudaSetDevice(c->device);
    dfree(c, key);
    dfree(c, parent);
    dfree(c, child0);
    dfree(c, coef);
    dfree(c, norm2);
    dfree(c, wnorm2);
    dfree(c, hkey);
    dfree(c, hval);
    cudaStreamSynchronize(c->stream);
}

void tree_reserve(Tree& t, int need) {
    Ctx* ctx = t.mra->ctx;
    cudaStream_t s = ctx->stream;
    if (need > t.cap) {
        int ncap = std::max(need, std::max(64, t.cap * 2));
        const size_t BS = t.mra->bsize();
        auto grow = [&](auto*& p, size_t elem) {
            using T = std::remove_reference_t<decltype(*p)>;
            T* q = (T*)dalloc(ctx, elem * ncap);
            if (p && t.n > 0) device_copy(ctx, q, p, elem * t.n);  // on s (= the context's stream)
            dfree(ctx, p);
            p = q;
        };
        grow(t.key, sizeof(uint64_t));
        grow(t.parent, sizeof(int));
        grow(t.child0, sizeof(int));
        grow(t.coef, sizeof(double) * BS);
        grow(t.norm2, sizeof(double));
        grow(t.wnorm2, sizeof(double));
        t.cap = ncap;
    }
    // hash index at most half full
    uint32_t hneed = 1024;
    while (hneed < 2u * (uint32_t)std::max(need, 1)) hneed <<= 1;
    if (hneed > t.hcap) {
        dfree(ctx, t.hkey);
        dfree(ctx, t.hval);
        t.hcap = hneed;
        t.hkey = (uint64_t*)dalloc(ctx, sizeof(uint64_t) * t.hcap);
        t.hval = (int*)dalloc(ctx, sizeof(int) * t.hcap);
        launch_hash_reset(t, s);
        launch_hash_insert(t, 0, t.n, s);
    }
}

// root boxes in Morton order
void tree_make_roots(Tree& t) {
    const Mra& m = *t.mra;
    std::vector<uint64_t> keys;
    for (int z = 0; z < m.boxes[2]; ++z)
        for (int y = 0; y < m.boxes[1]; ++y)
            for (int x = 0; x < m.boxes[0]; ++x) keys.push_back(host_make_key(0, x, y, z));
    std::sort(keys.begin(), keys.end());
    t.n = 0;
    t.level_begin.clear();
    tree_reserve(t, (int)keys.size());
    cudaStream_t s = m.ctx->stream;
    launch_hash_reset(t, s);
    const int n = (int)keys.size();
    std::vector<int> par(n, -1);
    upload_bytes(m.ctx, t.key, keys.data(), sizeof(uint64_t) * n);  // staged: the host vectors may go
    upload_bytes(m.ctx, t.parent, par.data(), sizeof(int) * n);
    upload_bytes(m.ctx, t.child0, par.data(), sizeof(int) * n);
    MWB_CUDA(cudaMemsetAsync(t.norm2, 0, sizeof(double) * n, s));
    MWB_CUDA(cudaMemsetAsync(t.wnorm2, 0, sizeof(double) * n, s));
    t.n = n;
    t.level_begin = {0, n};
    launch_hash_insert(t, 0, n, s);
}

// split the nodes of the last level whose wavelet norm exceeds thr; returns the number of new nodes
int tree_refine_last_level(Tree& t, double thr) {
    Ctx* ctx = t.mra->ctx;
    cudaStream_t s = ctx->stream;
    const int b = t.level_begin[t.levels() - 1], e = t.level_begin[t.levels()];
    const int depth = t.levels() - 1;
    int* d_list = (int*)dalloc(ctx, sizeof(int) * std::max(1, e - b));
    int ns = launch_split(t, b, e, depth, thr, t.mra->depth_limit, d_list, s);
    if (ns > 0) {
        tree_reserve(t, t.n + 8 * ns);
        launch_make_children(t, d_list, ns, s);
        launch_hash_insert(t, t.n, t.n + 8 * ns, s);
        t.n += 8 * ns;
        t.level_begin.push_back(t.n);
    }
    dfree(ctx, d_list);
    return 8 * ns;
}

static int* range_list(Ctx* ctx, int begin, int end) {
    std::vector<int> v(end - begin);
    std::iota(v.begin(), v.end(), begin);
    int* d = (int*)dalloc(ctx, sizeof(int) * std::max<size_t>(1, v.size()));
    MWB_CUDA(cudaMemcpyAsync(d, v.data(), sizeof(int) * v.size(), cudaMemcpyHostToDevice, ctx->stream));
    MWB_CUDA(cudaStreamSynchronize(ctx->stream));
    return d;
}

// bottom-up: every internal node becomes the compression of its children's scaling parts
void tree_compress_bottom_up(Tree& t) {
    cudaStream_t s = t.mra->ctx->stream;
    for (int d = t.levels() - 2; d >= 0; --d) {
        const int b = t.level_begin[d], e = t.level_begin[d + 1];
        launch_transform_nodes(t, TM_COMPRESS, nullptr, e - b, nullptr, s, b);
    }
}

// ---------------------------------------------------------------------------------------------
// projection
// ---------------------------------------------------------------------------------------------

static void project(double prec, Tree& t, int type, int np, const double* params) {
    Ctx* ctx = t.mra->ctx;
    cudaStream_t s = ctx->stream;
    if (np < 1) throw Error(MW_ERR_ARG, "empty parameter block");
    const int nterm = (int)params[0];
    const int per = (type == MW_FUNC_GAUSSIANS) ? 8 : (type == MW_FUNC_HYDROGEN_PRODUCTS ? 11 : -1);
    if (per < 0) throw Error(MW_ERR_ARG, "unknown function type");
    if (np < 1 + per * nterm) throw Error(MW_ERR_ARG, "parameter block too short");
    double* d_p = (double*)dalloc(ctx, sizeof(double) * np);
    MWB_CUDA(cudaMemcpyAsync(d_p, params, sizeof(double) * np, cudaMemcpyHostToDevice, s));
    FuncDesc f{type, nterm, d_p};
    tree_make_roots(t);
    int b = 0, e = t.n;
    while (e > b) {
        int* d_list = range_list(ctx, b, e);
        launch_transform_nodes(t, TM_PROJECT, d_list, e - b, &f, s);
        dfree(ctx, d_list);
        if (prec <= 0.0) break;
        const double ref = std::sqrt(reduce_leaf_norm2(t, s));
        const int added = tree_refine_last_level(t, split_threshold(prec, ref, t.levels() - 1));
        if (added == 0) break;
        b = e;
        e = t.n;
    }
    tree_compress_bottom_up(t);
    launch_node_norms(t, 0, t.n, s);
    MWB_CUDA(cudaStreamSynchronize(s));
    dfree(ctx, d_p);
}

// ---------------------------------------------------------------------------------------------
// operators
// ---------------------------------------------------------------------------------------------

Op::~Op() {
    if (!mra) return;
    Ctx* c = mra->ctx;
    cudaSetDevice(c->device);
    for (auto& kv : depths) {
        dfree(c, kv.second->d_mats);
        dfree(c, kv.second->d_mats32);
        dfree(c, kv.second->d_matsb);
        dfree(c, kv.second->d_matsb32);
        dfree(c, kv.second->d_matsT);
        dfree(c, kv.second->d_matsT32);
        dfree(c, kv.second->d_matsbT);
        dfree(c, kv.second->d_matsbT32);
        dfree(c, kv.second->d_matsI);
        dfree(c, kv.second->d_matsbI);
        dfree(c, kv.second->d_matsS32);
        dfree(c, kv.second->d_matsbS32);
        dfree(c, kv.second->d_matsX);
        dfree(c, kv.second->d_deltas);
        dfree(c, kv.second->d_terms);
    }
    cudaStreamSynchronize(c->stream);
}

struct BandTmp {
    bool active = false;
    int L = -1;
    std::vector<double> ns;  // l = -L..L
    std::vector<double> t2, x2;
};

static std::vector<BandTmp> op_bands(Op& op, int depth) {
    const Mra& m = *op.mra;
    const int k = m.k, K2 = 2 * k, n = m.n0 + depth;
    long extent = 0;
    for (int d = 0; d < 3; ++d) extent = std::max<long>(extent, (long)m.boxes[d] << depth);
    const double cut = depth == 0 ? 0.0 : 1e-6 * op.eps * op.B0 * std::pow(4.0, -depth);
    std::vector<BandTmp> bs(op.terms.size());
    for (size_t mi = 0; mi < op.terms.size(); ++mi) {
        BandTmp& b = bs[mi];
        std::vector<std::pair<long, std::vector<double>>> cache;
        std::vector<std::vector<double>> mats;
        std::vector<double> t2, x2;
        auto compute = [&](long l) {
            std::vector<double> NS(K2 * K2);
            op.builder->ns(op.terms[mi].alpha, n, l, NS.data(), cache);
            double tt = 0.0, xx = 0.0;
            for (int a = 0; a < K2; ++a)
                for (int c = 0; c < K2; ++c) {
                    const double v = NS[a * K2 + c] * NS[a * K2 + c];
                    if (a < k && c < k) tt += v; else xx += v;
                }
            mats.push_back(std::move(NS));
            t2.push_back(tt);
            x2.push_back(xx);
        };
        compute(0);
        compute(1);
        const double beta = op.terms[mi].beta;
        double S2 = std::max(t2[0] + x2[0], t2[1] + x2[1]);
        if (depth > 0) {
            const double xmax = std::sqrt(std::max(x2[0], x2[1]));
            if (beta * 10.0 * xmax * S2 < cut) continue;
        }
        long L = 1;
        while (L + 1 < extent) {
            const double last = std::sqrt(t2[L] + x2[L]);
            if (depth > 0 && beta * last * S2 < cut) break;
            if (depth == 0 && last <= 1e-300) break;
            if (depth == 0 && last < 1e-17 * std::sqrt(S2)) break;
            compute(L + 1);
            S2 = std::max(S2, t2[L + 1] + x2[L + 1]);
            ++L;
        }
        while (L > 0 && depth > 0 && beta * std::sqrt(t2[L] + x2[L]) * S2 < cut) --L;
        if (L >= extent) L = extent - 1;
        b.active = true;
        b.L = (int)L;
        b.ns.assign((size_t)(2 * L + 1) * K2 * K2, 0.0);
        b.t2.assign(2 * L + 1, 0.0);
        b.x2.assign(2 * L + 1, 0.0);
        for (long l = -L; l <= L; ++l) {
            const long al = l < 0 ? -l : l;
            double* dst = &b.ns[(size_t)(l + L) * K2 * K2];
            const std::vector<double>& src = mats[al];
            for (int a = 0; a < K2; ++a)
                for (int c = 0; c < K2; ++c) dst[a * K2 + c] = (l >= 0) ? src[a * K2 + c] : src[c * K2 + a];
            b.t2[l + L] = t2[al];
            b.x2[l + L] = x2[al];
        }
    }
    return bs;
}

static double bound3(double beta, const double* t, const double* x, bool root) {
    if (root) return beta * std::sqrt((t[0] + x[0]) * (t[1] + x[1]) * (t[2] + x[2]));
    const double v = x[0] * (t[1] + x[1]) * (t[2] + x[2]) + t[0] * x[1] * (t[2] + x[2]) + t[0] * t[1] * x[2];
    return beta * std::sqrt(v);
}

// Tables of a first-derivative operator along `dir` at one depth: one term (beta = 1) whose factor
// along `dir` is the derivative's NS matrix for the offset and the identity along the other two
// directions; offsets -1, 0, 1 along `dir`.  The NS matrix of offset l at scale n is
// F [[T(2l) T(2l-1)]; [T(2l+1) T(2l)]] F^T with T(d) = 2^{n+1} T_unit(d) at the children's scale.
static void derivative_depth(Op& op, int depth, int dir, OpDepth& od, std::vector<double>& mbeta) {
    const Mra& m = *op.mra;
    const int k = m.k, K2 = 2 * k;
    const double fac = std::ldexp(1.0, m.n0 + depth + 1);
    auto Tc = [&](int d, int i, int j) -> double {  // children-scale block T(d)[i][j]
        return (d < -1 || d > 1) ? 0.0 : fac * op.dT[d + 1][(size_t)i * k + j];
    };
    std::vector<double> ident((size_t)K2 * K2, 0.0);
    for (int a = 0; a < K2; ++a) ident[(size_t)a * K2 + a] = 1.0;
    od.mats = ident;  // matrix 0: identity
    double tn[3], xn[3];
    const double ti = (double)k, xi = (double)k;  // identity: k ones in the s-s block, k elsewhere
    for (int l = -1; l <= 1; ++l) {
        std::vector<double> C((size_t)K2 * K2, 0.0), tmp((size_t)K2 * K2, 0.0), NS((size_t)K2 * K2, 0.0);
        for (int co = 0; co < 2; ++co)
            for (int ci = 0; ci < 2; ++ci)
                for (int i = 0; i < k; ++i)
                    for (int j = 0; j < k; ++j) C[(size_t)(co * k + i) * K2 + ci * k + j] = Tc(2 * l + co - ci, i, j);
        for (int a = 0; a < K2; ++a)
            for (int c = 0; c < K2; ++c) {
                double v = 0.0;
                for (int b = 0; b < K2; ++b) v += m.F[(size_t)a * K2 + b] * C[(size_t)b * K2 + c];
                tmp[(size_t)a * K2 + c] = v;
            }
        double t2 = 0.0, x2 = 0.0;
        for (int a = 0; a < K2; ++a)
            for (int c = 0; c < K2; ++c) {
                double v = 0.0;
                for (int b = 0; b < K2; ++b) v += tmp[(size_t)a * K2 + b] * m.F[(size_t)c * K2 + b];
                NS[(size_t)a * K2 + c] = v;
                (a < k && c < k ? t2 : x2) += v * v;
            }
        tn[l + 1] = t2;
        xn[l + 1] = x2;
        od.mats.insert(od.mats.end(), NS.begin(), NS.end());  // matrix 2 + l
    }
    const bool root = depth == 0;
    std::vector<std::pair<DeltaRec, TermRec>> rows;
    for (int l = -1; l <= 1; ++l) {
        double t[3], x[3];
        for (int d = 0; d < 3; ++d) {
            t[d] = d == dir ? tn[l + 1] : ti;
            x[d] = d == dir ? xn[l + 1] : xi;
        }
        const double bd = bound3(1.0, t, x, root);
        if (!(bd > 0.0)) continue;
        DeltaRec dr{};
        dr.d[dir] = l;
        dr.maxb = bd;
        TermRec tr{};
        tr.m = 0;
        tr.mx = dir == 0 ? 2 + l : 0;
        tr.my = dir == 1 ? 2 + l : 0;
        tr.mz = dir == 2 ? 2 + l : 0;
        tr.beta = 1.0;
        tr.bound = bd;
        rows.emplace_back(dr, tr);
    }
    std::stable_sort(rows.begin(), rows.end(), [](const auto& a, const auto& b) { return a.first.maxb > b.first.maxb; });
    for (auto& r : rows) {
        r.first.t0 = (int)od.terms.size();
        od.terms.push_back(r.second);
        r.first.t1 = (int)od.terms.size();
        od.deltas.push_back(r.first);
    }
    mbeta.assign(4, 1.0);
}

// build (once) and upload the tables of one depth
static const OpDepth& op_depth(Op& op, int depth, int dir = 0) {
    std::lock_guard<std::mutex> g(op.mtx);
    const int ckey = op.kind == 1 ? 3 * depth + dir : depth;
    auto it = op.depths.find(ckey);
    if (it != op.depths.end()) return *it->second;
    const Mra& m = *op.mra;
    const int K2 = 2 * m.k;
    auto od = std::make_unique<OpDepth>();
    std::vector<double> mbeta;  // the term weight of every stored matrix (z-step tables)
    if (op.kind == 1) {
        derivative_depth(op, depth, dir, *od, mbeta);
    } else {
    std::vector<BandTmp> bs = op_bands(op, depth);
    std::vector<int> base(bs.size(), -1);
    for (size_t mi = 0; mi < bs.size(); ++mi) {
        if (!bs[mi].active) continue;
        base[mi] = (int)(od->mats.size() / (K2 * K2));
        od->mats.insert(od->mats.end(), bs[mi].ns.begin(), bs[mi].ns.end());
    }
    const bool root = depth == 0;
    const double cut = root ? 0.0 : 1e-6 * op.eps * op.B0 * std::pow(4.0, -depth);
    std::map<std::tuple<int, int, int>, std::vector<std::pair<double, int>>> acc;
    for (size_t mi = 0; mi < bs.size(); ++mi) {
        const BandTmp& b = bs[mi];
        if (!b.active) continue;
        const double beta = op.terms[mi].beta;
        double S2 = 0.0;
        for (int i = 0; i < 2 * b.L + 1; ++i) S2 = std::max(S2, b.t2[i] + b.x2[i]);
        for (int dx = -b.L; dx <= b.L; ++dx) {
            const double ax = b.t2[dx + b.L] + b.x2[dx + b.L];
            if (!root && beta * std::sqrt(ax) * S2 < cut) continue;
            for (int dy = -b.L; dy <= b.L; ++dy) {
                const double ay = b.t2[dy + b.L] + b.x2[dy + b.L];
                if (!root && beta * std::sqrt(ax * ay * S2) < cut) continue;
                for (int dz = -b.L; dz <= b.L; ++dz) {
                    const double t[3] = {b.t2[dx + b.L], b.t2[dy + b.L], b.t2[dz + b.L]};
                    const double x[3] = {b.x2[dx + b.L], b.x2[dy + b.L], b.x2[dz + b.L]};
                    const double bd = bound3(beta, t, x, root);
                    if (bd <= 0.0 || bd < cut) continue;
                    acc[std::make_tuple(dx, dy, dz)].push_back({bd, (int)mi});
                }
            }
        }
    }
    std::vector<std::pair<DeltaRec, std::vector<TermRec>>> rows;
    rows.reserve(acc.size());
    for (auto& kv : acc) {
        auto& v = kv.second;
        std::stable_sort(v.begin(), v.end(), [](const std::pair<double, int>& a, const std::pair<double, int>& b) {
            return a.first > b.first || (a.first == b.first && a.second < b.second);
        });
        DeltaRec dr{};
        dr.d[0] = std::get<0>(kv.first);
        dr.d[1] = std::get<1>(kv.first);
        dr.d[2] = std::get<2>(kv.first);
        dr.maxb = v.front().first;
        std::vector<TermRec> trs;
        for (auto& pr : v) {
            const int mi = pr.second;
            const BandTmp& b = bs[mi];
            TermRec tr{};
            tr.m = mi;
            tr.mx = base[mi] + dr.d[0] + b.L;
            tr.my = base[mi] + dr.d[1] + b.L;
            tr.mz = base[mi] + dr.d[2] + b.L;
            tr.beta = op.terms[mi].beta;
            tr.bound = pr.first;
            trs.push_back(tr);
        }
        rows.emplace_back(dr, std::move(trs));
    }
    std::stable_sort(rows.begin(), rows.end(),
                     [](const auto& a, const auto& b) { return a.first.maxb > b.first.maxb; });
    for (auto& r : rows) {
        r.first.t0 = (int)od->terms.size();
        od->terms.insert(od->terms.end(), r.second.begin(), r.second.end());
        r.first.t1 = (int)od->terms.size();
        od->deltas.push_back(r.first);
    }
    mbeta.assign(od->mats.size() / ((size_t)K2 * K2), 0.0);
    for (size_t mi = 0; mi < bs.size(); ++mi) {
        if (!bs[mi].active) continue;
        for (int q = 0; q < 2 * bs[mi].L + 1; ++q) mbeta[base[mi] + q] = op.terms[mi].beta;
    }
    }
    // line ranks: the contraction groups an output node's triples by (term, dz, dy) (sort key bits:
    // term << 20 | dz rank << 10 | dy rank), so that the triples of one line share their y and z steps
    {
        std::vector<int> zs, ys;
        for (const DeltaRec& d : od->deltas) {
            zs.push_back(d.d[2]);
            ys.push_back(d.d[1]);
        }
        for (auto* v : {&zs, &ys}) {
            std::sort(v->begin(), v->end());
            v->erase(std::unique(v->begin(), v->end()), v->end());
        }
        if (zs.size() > 1024 || ys.size() > 1024)
            throw Error(MW_ERR_CAPACITY, "operator band wider than 1024 offsets per direction");
        for (DeltaRec& d : od->deltas) {
            const int rz = (int)(std::lower_bound(zs.begin(), zs.end(), d.d[2]) - zs.begin());
            const int ry = (int)(std::lower_bound(ys.begin(), ys.end(), d.d[1]) - ys.begin());
            d.lrank = (rz << 10) | ry;
        }
        for (const TermRec& t : od->terms)
            if (t.m < 0 || t.m >= 4096) throw Error(MW_ERR_CAPACITY, "more than 4096 operator terms");
    }
    Ctx* ctx = m.ctx;
    cudaStream_t s = ctx->stream;
    od->d_mats = (double*)dalloc(ctx, sizeof(double) * std::max<size_t>(1, od->mats.size()));
    od->d_deltas = (DeltaRec*)dalloc(ctx, sizeof(DeltaRec) * std::max<size_t>(1, od->deltas.size()));
    od->d_terms = (TermRec*)dalloc(ctx, sizeof(TermRec) * std::max<size_t>(1, od->terms.size()));
    od->d_mats32 = (float*)dalloc(ctx, sizeof(float) * std::max<size_t>(1, od->mats.size()));
    od->d_matsb = (double*)dalloc(ctx, sizeof(double) * std::max<size_t>(1, od->mats.size()));
    od->d_matsb32 = (float*)dalloc(ctx, sizeof(float) * std::max<size_t>(1, od->mats.size()));
    std::vector<float> m32(od->mats.begin(), od->mats.end());
    std::vector<double> mb(od->mats.size());
    for (size_t q = 0; q < od->mats.size(); ++q) mb[q] = mbeta[q / ((size_t)K2 * K2)] * od->mats[q];
    std::vector<float> mb32(mb.begin(), mb.end());
    // transposed, zero-padded copies for the GEMM-tiled contraction
    const int KP = (K2 + 3) / 4 * 4;
    const size_t nmat = od->mats.size() / ((size_t)K2 * K2);
    std::vector<double> mT(nmat * KP * KP, 0.0), mbT(nmat * KP * KP, 0.0);
    for (size_t mi = 0; mi < nmat; ++mi)
        for (int o = 0; o < K2; ++o)
            for (int k = 0; k < K2; ++k) {
                mT[mi * KP * KP + (size_t)k * KP + o] = od->mats[mi * K2 * K2 + (size_t)o * K2 + k];
                mbT[mi * KP * KP + (size_t)k * KP + o] = mb[mi * K2 * K2 + (size_t)o * K2 + k];
            }
    std::vector<float> mT32(mT.begin(), mT.end()), mbT32(mbT.begin(), mbT.end());
    od->d_matsT = (double*)dalloc(ctx, sizeof(double) * std::max<size_t>(1, mT.size()));
    od->d_matsT32 = (float*)dalloc(ctx, sizeof(float) * std::max<size_t>(1, mT.size()));
    od->d_matsbT = (double*)dalloc(ctx, sizeof(double) * std::max<size_t>(1, mT.size()));
    od->d_matsbT32 = (float*)dalloc(ctx, sizeof(float) * std::max<size_t>(1, mT.size()));
    // split-TF32 images: three TF32 pieces per entry (hi, mid, lo: each the TF32 rounding of what the
    // previous pieces leave of the FP64 value)
    const int KP8 = (K2 + 7) / 8 * 8;
    const size_t isz = (size_t)3 * KP8 * KP8;
    std::vector<float> mI(nmat * isz, 0.0f), mbI(nmat * isz, 0.0f);
    auto put3 = [&](std::vector<float>& img, size_t mi, int o, int k, double v) {
        const size_t w = mi * isz + (size_t)(o + 3 * KP8 * (k / 4)) * 4 + k % 4;  // row o of the hi block
        const float h = tf32_round((float)v);
        const float md = tf32_round((float)(v - (double)h));
        const float l = tf32_round((float)(v - (double)h - (double)md));
        img[w] = h;
        img[w + 4 * (size_t)KP8] = md;  // row KP8 + o
        img[w + 8 * (size_t)KP8] = l;   // row 2 KP8 + o
    };
    for (size_t mi = 0; mi < nmat; ++mi)
        for (int o = 0; o < K2; ++o)
            for (int k = 0; k < K2; ++k) {
                put3(mI, mi, o, k, od->mats[mi * K2 * K2 + (size_t)o * K2 + k]);
                put3(mbI, mi, o, k, mb[mi * K2 * K2 + (size_t)o * K2 + k]);
            }
    od->d_matsI = (float*)dalloc(ctx, sizeof(float) * std::max<size_t>(1, mI.size()));
    od->d_matsbI = (float*)dalloc(ctx, sizeof(float) * std::max<size_t>(1, mI.size()));
    if (!mI.empty()) {
        MWB_CUDA(cudaMemcpyAsync(od->d_matsI, mI.data(), sizeof(float) * mI.size(), cudaMemcpyHostToDevice, s));
        MWB_CUDA(cudaMemcpyAsync(od->d_matsbI, mbI.data(), sizeof(float) * mbI.size(), cudaMemcpyHostToDevice, s));
    }
    // tensor-core x step (k_happly, 2k <= 20): split-layout FP32 operators of the y/z tiles and the BF16
    // slice images of every matrix as an x operator
    if (K2 >= 13 && K2 <= 20) {
        const int MT = KP / 4;
        std::vector<float> mS(nmat * KP * KP, 0.0f), mbS(nmat * KP * KP, 0.0f);
        for (size_t mi = 0; mi < nmat; ++mi)
            for (int o = 0; o < K2; ++o)
                for (int k = 0; k < K2; ++k) {
                    const size_t w = mi * KP * KP + (size_t)k * KP + split_pos(o, MT, 4);
                    mS[w] = (float)od->mats[mi * K2 * K2 + (size_t)o * K2 + k];
                    mbS[w] = (float)mb[mi * K2 * K2 + (size_t)o * K2 + k];
                }
        const XGeo xg(K2);
        std::vector<uint16_t> mX(nmat * (size_t)xg.OPB / 2, 0);
        std::vector<float> sl0(K2), sl1(K2), sl2(K2), t0(K2), t1(K2), t2(K2);
        for (size_t mi = 0; mi < nmat; ++mi) {
            uint16_t* img = mX.data() + mi * (size_t)xg.OPB / 2;
            for (int o = 0; o < K2; ++o) {
                slice3_row(&od->mats[mi * K2 * K2 + (size_t)o * K2], K2, 1, sl0.data(), sl1.data(), sl2.data());
                const float* sl[3] = {sl0.data(), sl1.data(), sl2.data()};
                if (o < xg.W2)  // the s->s block row M[o][0 .. k)
                    slice3_row(&od->mats[mi * K2 * K2 + (size_t)o * K2], xg.W2, 1, t0.data(), t1.data(), t2.data());
                const float* tl[3] = {t0.data(), t1.data(), t2.data()};
                for (int q = 0; q < 3; ++q) {  // (a) the operand of data slice q
                    uint16_t* op = img + (size_t)q * xg.OPB_Q / 2;
                    for (int b = q; b < 3; ++b) {
                        const int row = b * xg.W + o;
                        for (int k = 0; k < std::min(K2, 8 * xg.NCHM); ++k)
                            op[((size_t)(k / 8) * xg.NBQ + row) * 8 + k % 8] = bf16_bits_exact(sl[b - q][k]);
                        if (o < xg.W2) {
                            const int row2 = xg.NCOL + b * xg.W2 + o;
                            for (int k = 0; k < xg.W2; ++k)
                                op[((size_t)(k / 8) * xg.NBQ + row2) * 8 + k % 8] = bf16_bits_exact(tl[b - q][k]);
                        }
                    }
                }
                if (xg.PACK) {  // (b) the packed step over x = 16 .. K2-1
                    uint16_t* pk = img + (size_t)xg.OPB_A / 2;
                    for (int b = 0; b < 3; ++b)
                        for (int q = 0; q <= b; ++q)
                            for (int l = 0; l < xg.LO; ++l) {
                                const int kk = 4 * q + l, row = b * xg.W + o;
                                pk[((size_t)(kk / 8) * xg.NCOL + row) * 8 + kk % 8] = bf16_bits_exact(sl[b - q][16 + l]);
                            }
                    for (int l = 0; l < xg.LO; ++l) {  // data slice 3 against operator slice 0, into block 2
                        const int kk = 12 + l, row = 2 * xg.W + o;
                        pk[((size_t)(kk / 8) * xg.NCOL + row) * 8 + kk % 8] = bf16_bits_exact(sl[0][16 + l]);
                    }
                }
            }
        }
        od->d_matsS32 = (float*)dalloc(ctx, sizeof(float) * std::max<size_t>(1, mS.size()));
        od->d_matsbS32 = (float*)dalloc(ctx, sizeof(float) * std::max<size_t>(1, mS.size()));
        od->d_matsX = (unsigned char*)dalloc(ctx, std::max<size_t>(16, mX.size() * 2));
        if (!mS.empty()) {
            MWB_CUDA(cudaMemcpyAsync(od->d_matsS32, mS.data(), sizeof(float) * mS.size(), cudaMemcpyHostToDevice, s));
            MWB_CUDA(cudaMemcpyAsync(od->d_matsbS32, mbS.data(), sizeof(float) * mS.size(), cudaMemcpyHostToDevice, s));
            MWB_CUDA(cudaMemcpyAsync(od->d_matsX, mX.data(), mX.size() * 2, cudaMemcpyHostToDevice, s));
        }
        MWB_CUDA(cudaStreamSynchronize(s));  // host vectors leave scope
    }
    if (!mT.empty()) {
        MWB_CUDA(cudaMemcpyAsync(od->d_matsT, mT.data(), sizeof(double) * mT.size(), cudaMemcpyHostToDevice, s));
        MWB_CUDA(cudaMemcpyAsync(od->d_matsT32, mT32.data(), sizeof(float) * mT.size(), cudaMemcpyHostToDevice, s));
        MWB_CUDA(cudaMemcpyAsync(od->d_matsbT, mbT.data(), sizeof(double) * mT.size(), cudaMemcpyHostToDevice, s));
        MWB_CUDA(cudaMemcpyAsync(od->d_matsbT32, mbT32.data(), sizeof(float) * mT.size(), cudaMemcpyHostToDevice, s));
    }
    if (!od->mats.empty()) {
        MWB_CUDA(cudaMemcpyAsync(od->d_mats, od->mats.data(), sizeof(double) * od->mats.size(), cudaMemcpyHostToDevice, s));
        MWB_CUDA(cudaMemcpyAsync(od->d_mats32, m32.data(), sizeof(float) * m32.size(), cudaMemcpyHostToDevice, s));
        MWB_CUDA(cudaMemcpyAsync(od->d_matsb, mb.data(), sizeof(double) * mb.size(), cudaMemcpyHostToDevice, s));
        MWB_CUDA(cudaMemcpyAsync(od->d_matsb32, mb32.data(), sizeof(float) * mb32.size(), cudaMemcpyHostToDevice, s));
    }
    if (!od->deltas.empty())
        MWB_CUDA(cudaMemcpyAsync(od->d_deltas, od->deltas.data(), sizeof(DeltaRec) * od->deltas.size(), cudaMemcpyHostToDevice, s));
    if (!od->terms.empty())
        MWB_CUDA(cudaMemcpyAsync(od->d_terms, od->terms.data(), sizeof(TermRec) * od->terms.size(), cudaMemcpyHostToDevice, s));
    MWB_CUDA(cudaStreamSynchronize(s));
    return *op.depths.emplace(ckey, std::move(od)).first->second;
}

static void op_init(Op& op, Mra* m, double mu, double prec) {
    if (!(prec > 0.0)) throw Error(MW_ERR_ARG, "operator precision must be positive");
    if (mu < 0.0) throw Error(MW_ERR_ARG, "mu must be non-negative");
    op.mra = m;
    op.mu = mu;
    op.prec = prec;
    op.eps = 0.1 * prec;
    const double root_edge = std::ldexp(1.0, -m->n0);
    double r_max = 0.0;
    for (int d = 0; d < 3; ++d) r_max += std::pow(m->boxes[d] * root_edge, 2);
    r_max = std::sqrt(r_max);
    const double r_min = 0.01 * std::ldexp(root_edge, -m->max_depth);
    op.terms = kernel_expansion(mu, op.eps, r_min, r_max);
    op.builder = std::make_unique<GaussianOperatorBuilder>(m->basis, m->F);
    // operator scale from the root-depth bands
    std::vector<BandTmp> b0 = op_bands(op, 0);
    op.B0 = 0.0;
    for (size_t mi = 0; mi < op.terms.size(); ++mi) {
        if (!b0[mi].active) continue;
        const int L = b0[mi].L;
        op.B0 = std::max(op.B0, op.terms[mi].beta * std::pow(b0[mi].t2[L] + b0[mi].x2[L], 1.5));
    }
}

// ---------------------------------------------------------------------------------------------
// apply
// ---------------------------------------------------------------------------------------------

// append the 8 children of every listed node, for several trees, with one synchronisation
static void add_children_many(const std::vector<Tree*>& ts, const std::vector<std::vector<int>>& lists) {
    if (ts.empty()) return;
    trees_add_children(ts, lists, ts[0]->mra->ctx->stream);
}


// Adaptive NS-form apply of a batch: out[i] = op[i] * inp[i], all trees on one world.  The passes
// run in lock-step over the batch (one launch per stage for all trees of a depth).
static void apply_batched(double prec, int n, Tree** out, Op** op, Tree** inp, int precision) {
    if (n <= 0) throw Error(MW_ERR_ARG, "empty batch");
    for (int i = 0; i < n; ++i)
        if (op[i] && op[i]->kind != 0) throw Error(MW_ERR_ARG, "derivative operators are applied with mw_apply_derivative");
    if (n > 128) throw Error(MW_ERR_ARG, "at most 128 trees per batch");
    const Mra* m = inp[0]->mra;
    for (int i = 0; i < n; ++i) {
        if (!out[i] || !op[i] || !inp[i]) throw Error(MW_ERR_ARG, "null tree or operator");
        if (out[i]->mra != m || inp[i]->mra != m || op[i]->mra != m)
            throw Error(MW_ERR_ARG, "trees and operators must share the world");
        if (inp[i]->n == 0) throw Error(MW_ERR_STATE, "input tree is empty");
        for (int j = 0; j < n; ++j)
            if (out[i] == inp[j] || (j != i && out[i] == out[j]))
                throw Error(MW_ERR_ARG, "output trees must be distinct from each other and from the inputs");
    }
    Ctx* ctx = m->ctx;
    cudaStream_t s = ctx->stream;
    std::vector<double> fnorm(n), nu_max(n), g0(n, 0.0);
    long long total_trip = 0;
    std::vector<int> passes(n, 0);
    std::vector<bool> active(n, true);
    {
        std::vector<Tree*> ins(inp, inp + n);
        std::vector<double> l2, m2;
        reduce_norms_many(ins, l2, m2, s);
        trees_make_roots(std::vector<Tree*>(out, out + n));
        for (int i = 0; i < n; ++i) {
            fnorm[i] = std::sqrt(l2[i]);
            nu_max[i] = std::sqrt(m2[i]);
        }
    }
    for (int depth = 0;; ++depth) {
        BatchPass bp;
        bp.precision = precision;
        std::vector<int> idx;
        for (int i = 0; i < n; ++i) {
            if (!active[i] || out[i]->levels() <= depth) continue;
            const int b = out[i]->level_begin[depth], e = out[i]->level_begin[depth + 1];
            if (e <= b) continue;
            BatchTree bt;
            bt.out = out[i];
            bt.inp = inp[i];
            bt.tab = &op_depth(*op[i], depth);
            bt.obegin = b;
            bt.oend = e;
            bt.prec = prec;
            bt.g0 = g0[i];
            bt.depth = depth;
            if (depth == 0) {
                const double nu0 = bt.tab->deltas.empty() ? 0.0 : bt.tab->deltas.front().maxb;
                bt.theta = kScreen * prec * fnorm[i] * nu0;
            } else {
                bt.theta = kScreen * split_threshold(prec, g0[i], depth);
            }
            int np = 0;
            while (nu_max[i] > 0.0 && np < (int)bt.tab->deltas.size() && !(bt.tab->deltas[np].maxb * nu_max[i] < bt.theta))
                ++np;
            bt.nprefix = np;
            bp.trees.push_back(bt);
            idx.push_back(i);
        }
        if (bp.trees.empty()) break;
        run_batch_pass(bp, s);
        std::vector<Tree*> grow;
        std::vector<std::vector<int>> lists;
        for (size_t q = 0; q < idx.size(); ++q) {
            const int i = idx[q];
            ++passes[i];
            if (depth == 0) g0[i] = bp.trees[q].g0;
            if (!(prec > 0.0) || !(g0[i] > 0.0) || bp.split_lists[q].empty()) {
                active[i] = false;
                continue;
            }
            grow.push_back(out[i]);
            lists.push_back(bp.split_lists[q]);
        }
        add_children_many(grow, lists);
        total_trip += bp.triples;
    }
    trees_finish(std::vector<Tree*>(out, out + n), true, true, true, s);
    MWB_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < n; ++i) {
        out[i]->g0 = g0[i];
        out[i]->prec = prec;
        out[i]->stats[0] = (n == 1) ? total_trip : -1;
        out[i]->stats[1] = total_trip;
        out[i]->stats[2] = passes[i];
        out[i]->stats[3] = out[i]->n;
    }
}

// run passes over explicit (tree, depth, node range) entries, at most 128 entries per launch set
struct Entry {
    int tree, depth, begin, end;
};
static long long run_entries(double prec, int precision, const std::vector<Entry>& ents, Tree** out, Op** op,
                             Tree** inp, const std::vector<double>& fnorm, const std::vector<double>& nu_max,
                             const std::vector<double>& g0, int dir = 0) {
    long long trip = 0;
    cudaStream_t s = out[0]->mra->ctx->stream;
    for (size_t e0 = 0; e0 < ents.size(); e0 += 128) {
        BatchPass bp;
        bp.precision = precision;
        for (size_t e = e0; e < std::min(ents.size(), e0 + 128); ++e) {
            const Entry& en = ents[e];
            const int i = en.tree;
            BatchTree bt;
            bt.out = out[i];
            bt.inp = inp[i];
            bt.tab = &op_depth(*op[i], en.depth, dir);
            bt.obegin = en.begin;
            bt.oend = en.end;
            bt.prec = prec;
            bt.g0 = g0[i];
            bt.depth = en.depth;
            if (en.depth == 0) {
                const double nu0 = bt.tab->deltas.empty() ? 0.0 : bt.tab->deltas.front().maxb;
                bt.theta = kScreen * prec * fnorm[i] * nu0;
            } else {
                bt.theta = kScreen * split_threshold(prec, g0[i], en.depth);
            }
            int np = 0;
            while (nu_max[i] > 0.0 && np < (int)bt.tab->deltas.size() && !(bt.tab->deltas[np].maxb * nu_max[i] < bt.theta))
                ++np;
            bt.nprefix = np;
            bp.trees.push_back(bt);
        }
        run_batch_pass(bp, s);
        trip += bp.triples;
    }
    return trip;
}

// Learned apply: exact root pass, network proposal of the deeper tree, one pass over all proposed
// nodes, then the plain criterion on every computed node (prune extras, refine misses).  The output
// equals apply_batched's.  stats: [0] triples, [1] passes, [2] proposed nodes, [3] pruned,
// [4] missed (refined) splits, [5] output nodes
static void apply_learned(double prec, int n, Tree** out, Op** op, Tree** inp, int precision, Mlp& M, float tau,
                          long long* stats) {
    if (n <= 0 || n > 128) throw Error(MW_ERR_ARG, "batch size must be in [1, 128]");
    const Mra* m = inp[0]->mra;
    for (int i = 0; i < n; ++i) {
        if (!out[i] || !op[i] || !inp[i]) throw Error(MW_ERR_ARG, "null tree or operator");
        if (out[i]->mra != m || inp[i]->mra != m || op[i]->mra != m)
            throw Error(MW_ERR_ARG, "trees and operators must share the world");
        if (inp[i]->n == 0) throw Error(MW_ERR_STATE, "input tree is empty");
        for (int j = 0; j < n; ++j)
            if (out[i] == inp[j] || (j != i && out[i] == out[j]))
                throw Error(MW_ERR_ARG, "output trees must be distinct from each other and from the inputs");
    }
    if (!(prec > 0.0)) throw Error(MW_ERR_ARG, "the learned apply needs prec > 0");
    for (int i = 0; i < n; ++i)
        if (op[i]->kind != 0) throw Error(MW_ERR_ARG, "derivative operators are applied with mw_apply_derivative");
    Ctx* ctx = m->ctx;
    cudaStream_t s = ctx->stream;
    const float logit_tau = std::log(tau / (1.0f - tau));
    std::vector<double> fnorm(n), nu_max(n), g0(n, 0.0);
    long long trip = 0, proposed = 0, pruned = 0, missed = 0;
    int passes = 0;
    std::vector<Entry> ents;
    {
        std::vector<Tree*> ins(inp, inp + n);
        std::vector<double> l2, m2;
        reduce_norms_many(ins, l2, m2, s);
        trees_make_roots(std::vector<Tree*>(out, out + n));
        for (int i = 0; i < n; ++i) {
            fnorm[i] = std::sqrt(l2[i]);
            nu_max[i] = std::sqrt(m2[i]);
            ents.push_back(Entry{i, 0, 0, out[i]->n});
        }
    }
    // exact root pass (sets g0)
    {
        BatchPass bp;
        bp.precision = precision;
        for (const Entry& en : ents) {
            const int i = en.tree;
            BatchTree bt;
            bt.out = out[i];
            bt.inp = inp[i];
            bt.tab = &op_depth(*op[i], 0);
            bt.obegin = en.begin;
            bt.oend = en.end;
            bt.prec = prec;
            bt.depth = 0;
            const double nu0 = bt.tab->deltas.empty() ? 0.0 : bt.tab->deltas.front().maxb;
            bt.theta = kScreen * prec * fnorm[i] * nu0;
            int np = 0;
            while (nu_max[i] > 0.0 && np < (int)bt.tab->deltas.size() && !(bt.tab->deltas[np].maxb * nu_max[i] < bt.theta))
                ++np;
            bt.nprefix = np;
            bp.trees.push_back(bt);
        }
        run_batch_pass(bp, s);
        trip += bp.triples;
        ++passes;
        std::vector<Tree*> rt(out, out + n);
        std::vector<std::vector<int>> rl(n);
        for (int i = 0; i < n; ++i) {
            g0[i] = bp.trees[i].g0;
            if (g0[i] > 0.0) rl[i] = bp.split_lists[i];
        }
        add_children_many(rt, rl);
    }
    // proposal: level by level, the network decides which nodes will split
    std::vector<FeatCtx> fc(n);
    for (int i = 0; i < n; ++i) fc[i] = FeatCtx{out[i], inp[i], op[i], prec, g0[i]};
    std::vector<long long> budget_used(n, 0);
    std::vector<Tree*> all(out, out + n);
    for (int depth = 1;; ++depth) {
        std::vector<int2> items;
        for (int i = 0; i < n; ++i) {
            if (out[i]->levels() <= depth || depth >= m->depth_limit) continue;
            for (int q = out[i]->level_begin[depth]; q < out[i]->level_begin[depth + 1]; ++q) items.push_back(int2{i, q});
        }
        if (items.empty()) break;
        float* d_F = features(ctx, fc, items, s);
        std::vector<float> z = mlp_logits(M, d_F, (int)items.size(), s);
        dfree(ctx, d_F);
        std::vector<std::vector<int>> lists(n);
        for (size_t q = 0; q < items.size(); ++q)
            if (z[q] > logit_tau) lists[items[q].x].push_back(items[q].y);
        bool any = false;
        for (int i = 0; i < n; ++i) {
            // proposal budget: twice the input tree; what lies beyond is left to the exact refinement
            const long long room = 2LL * inp[i]->n - budget_used[i];
            if ((long long)lists[i].size() * 8 > room) lists[i].resize(std::max(0LL, room / 8));
            budget_used[i] += 8LL * (long long)lists[i].size();
            proposed += 8LL * (long long)lists[i].size();
            any |= !lists[i].empty();
        }
        if (!any) break;
        add_children_many(all, lists);
    }
    // compute every node below the root level in one pass set
    ents.clear();
    for (int i = 0; i < n; ++i)
        for (int d = 1; d < out[i]->levels(); ++d)
            if (out[i]->level_begin[d + 1] > out[i]->level_begin[d])
                ents.push_back(Entry{i, d, out[i]->level_begin[d], out[i]->level_begin[d + 1]});
    if (!ents.empty()) {
        trip += run_entries(prec, precision, ents, out, op, inp, fnorm, nu_max, g0);
        ++passes;
    }
    // exact criterion on every computed node (on the device): a node is kept when all its ancestors
    // split; nodes below a node the criterion does not split are dropped at the final rebuild, kept
    // splits without children (misses) are refined by further passes
    std::vector<std::vector<double>> thr(n, std::vector<double>(64, INFINITY));
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 64; ++d) thr[i][d] = split_threshold(prec, g0[i], d);
    unsigned char* d_keep = nullptr;
    for (;;) {
        long long tot = 0;
        for (int i = 0; i < n; ++i) tot += out[i]->n;
        dfree(ctx, d_keep);
        d_keep = (unsigned char*)dalloc(ctx, std::max<long long>(1, tot));
        const std::vector<Miss> ms = verify_trees(all, thr, m->depth_limit, d_keep, s);
        if (ms.empty()) break;
        // per tree, in key order (depth-major): the appended children come out grouped by depth
        std::vector<std::vector<std::pair<uint64_t, int>>> mk(n);
        for (const Miss& q : ms) mk[q.tree].push_back({q.key, q.node});
        std::vector<std::vector<int>> lists(n);
        for (int i = 0; i < n; ++i) {
            std::sort(mk[i].begin(), mk[i].end());
            for (auto& kv : mk[i]) lists[i].push_back(kv.second);
        }
        missed += (long long)ms.size();
        std::vector<int> base(n);
        for (int i = 0; i < n; ++i) base[i] = out[i]->n;
        add_children_many(all, lists);
        std::vector<Entry> next;
        for (int i = 0; i < n; ++i) {
            int b = base[i];
            for (size_t q = 0; q < mk[i].size();) {
                const int d = (int)(mk[i][q].first >> 59) + 1;
                size_t r = q;
                while (r < mk[i].size() && (int)(mk[i][r].first >> 59) + 1 == d) ++r;
                next.push_back(Entry{i, d, b, b + 8 * (int)(r - q)});
                b += 8 * (int)(r - q);
                q = r;
            }
        }
        trip += run_entries(prec, precision, next, out, op, inp, fnorm, nu_max, g0);
        ++passes;
    }
    // one rebuild of every tree from its kept nodes, in key order (drops pruned nodes, puts the
    // appended refinements in level order)
    pruned += trees_rebuild_device(all, d_keep, s);
    dfree(ctx, d_keep);
    trees_finish(std::vector<Tree*>(out, out + n), true, true, true, s);
    for (int i = 0; i < n; ++i) {
        out[i]->g0 = g0[i];
        out[i]->prec = prec;
        out[i]->stats[0] = n == 1 ? trip : -1;
        out[i]->stats[1] = trip;
        out[i]->stats[2] = passes;
        out[i]->stats[3] = out[i]->n;
    }
    MWB_CUDA(cudaStreamSynchronize(s));
    if (stats) {
        long long nout = 0;
        for (int i = 0; i < n; ++i) nout += out[i]->n;
        stats[0] = trip;
        stats[1] = passes;
        stats[2] = proposed;
        stats[3] = pruned;
        stats[4] = missed;
        stats[5] = nout;
    }
}

// out = d/dx_dir inp on the input's grid (no refinement, no screening): the output takes the input's
// nodes, every level is one entry of a single pass set, then sum-up, compression and norms.
static void apply_derivative(Tree* out, Op* op, Tree* inp, int dir, int precision) {
    if (!out || !op || !inp) throw Error(MW_ERR_ARG, "null tree or operator");
    if (op->kind != 1) throw Error(MW_ERR_ARG, "not a derivative operator");
    if (dir < 0 || dir > 2) throw Error(MW_ERR_ARG, "direction must be 0, 1 or 2");
    if (out->mra != inp->mra || op->mra != inp->mra) throw Error(MW_ERR_ARG, "trees and operator on different worlds");
    if (inp->n == 0) throw Error(MW_ERR_STATE, "input tree is empty");
    if (out == inp) throw Error(MW_ERR_ARG, "output tree is also the input");
    Ctx* ctx = inp->mra->ctx;
    cudaStream_t s = ctx->stream;
    // grid of the input
    out->n = 0;
    tree_reserve(*out, inp->n);
    MWB_CUDA(cudaMemcpyAsync(out->key, inp->key, sizeof(uint64_t) * inp->n, cudaMemcpyDeviceToDevice, s));
    MWB_CUDA(cudaMemcpyAsync(out->parent, inp->parent, sizeof(int) * inp->n, cudaMemcpyDeviceToDevice, s));
    MWB_CUDA(cudaMemcpyAsync(out->child0, inp->child0, sizeof(int) * inp->n, cudaMemcpyDeviceToDevice, s));
    out->n = inp->n;
    out->level_begin = inp->level_begin;
    launch_hash_reset(*out, s);
    launch_hash_insert(*out, 0, out->n, s);
    std::vector<Tree*> ins{inp};
    std::vector<double> l2, m2;
    reduce_norms_many(ins, l2, m2, s);
    std::vector<double> fnorm{std::sqrt(l2[0])}, nu_max{std::sqrt(m2[0])}, g0{0.0};
    std::vector<Entry> ents;
    for (int d = 0; d < out->levels(); ++d)
        if (out->level_begin[d + 1] > out->level_begin[d]) ents.push_back(Entry{0, d, out->level_begin[d], out->level_begin[d + 1]});
    Tree* o[1] = {out};
    Op* p[1] = {op};
    Tree* i1[1] = {inp};
    const long long trip = run_entries(0.0, precision, ents, o, p, i1, fnorm, nu_max, g0, dir);
    trees_finish(std::vector<Tree*>{out}, true, true, true, s);
    MWB_CUDA(cudaStreamSynchronize(s));
    out->g0 = 0.0;
    out->prec = 0.0;
    out->stats[0] = trip;
    out->stats[1] = trip;
    out->stats[2] = (long long)((ents.size() + 127) / 128);
    out->stats[3] = out->n;
}

// features and labels (split or not) of the non-root nodes of an applied output tree
static void collect_training(Mlp& M, Tree& out, Op& op, Tree& inp) {
    if (out.n == 0 || out.levels() < 2) return;
    Ctx* ctx = out.mra->ctx;
    cudaStream_t s = ctx->stream;
    std::vector<FeatCtx> fc{FeatCtx{&out, &inp, &op, out.prec, out.g0}};
    std::vector<int2> items;
    std::vector<int> c0(out.n);
    MWB_CUDA(cudaMemcpyAsync(c0.data(), out.child0, sizeof(int) * out.n, cudaMemcpyDeviceToHost, s));
    MWB_CUDA(cudaStreamSynchronize(s));
    std::vector<float> y;
    for (int q = out.level_begin[1]; q < out.n; ++q) {
        items.push_back(int2{0, q});
        y.push_back(c0[q] >= 0 ? 1.0f : 0.0f);
    }
    float* d_F = features(ctx, fc, items, s);
    mlp_append(M, d_F, y, s);
    dfree(ctx, d_F);
}

}  // namespace mwb

// =============================================================================================
// C-ABI
// =============================================================================================
using namespace mwb;

struct mw_ctx_s : Ctx {};
struct mw_mra_s : Mra {};
struct mw_tree_s : Tree {};
struct mw_op_s : Op {};
struct mw_mlp_s : Mlp {};

// Handle lifetimes: a context or world destroyed while handles still point to it is freed when the
// last of them goes, so the C-ABI's destroy calls may come in any order (e.g. from a garbage collector
// finalising a reference cycle).
static void ctx_free(mwb::Ctx* ctx) {
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->pin_ev) cudaEventDestroy(ctx->pin_ev);
    if (ctx->pin) cudaFreeHost(ctx->pin);
    if (ctx->mbox) cudaFreeHost(ctx->mbox);
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    delete static_cast<mw_ctx_s*>(ctx);
}
static void ctx_release(mwb::Ctx* ctx) {
    if (--ctx->refs == 0 && ctx->closed) ctx_free(ctx);
}
static void mra_free(mwb::Mra* m) {
    mwb::Ctx* c = m->ctx;
    cudaSetDevice(c->device);
    mwb::dfree(c, m->d_F);
    mwb::dfree(c, m->d_FT);
    mwb::dfree(c, m->d_PF);
    mwb::dfree(c, m->d_MV);
    cudaStreamSynchronize(c->stream);
    delete static_cast<mw_mra_s*>(m);
    ctx_release(c);
}
static void mra_release(mwb::Mra* m) {
    if (--m->refs == 0 && m->closed) mra_free(m);
}

#define MW_TRY(...)                                        \
    try {                                                  \
        __VA_ARGS__;                                       \
        return MW_OK;                                      \
    } catch (const mwb::Error& e) {                        \
        g_err = e.what();                                  \
        return e.code;                                     \
    } catch (const std::exception& e) {                    \
        g_err = e.what();                                  \
        return MW_ERR_STATE;                               \
    }

#define MW_ARG(cond, msg) \
    if (!(cond)) throw mwb::Error(MW_ERR_ARG, msg)

// Host half of a tree upload: checks, (depth, Morton) order (parents before children, siblings in child
// order), parent / child indices relinked to that order, level starts.
struct HostTree {
    int n = 0;
    bool sorted = true;
    std::vector<uint64_t> key;  // in (depth, Morton) order
    std::vector<int> parent, child0, ord, lb;
};
static void upload_prepare(const Mra& m, int n, const int* depth, const long long* trans, const int* parent,
                           const int* child0, HostTree& h) {
    std::vector<uint64_t> key(n);
    int maxd = 0;
    for (int i = 0; i < n; ++i) {
        MW_ARG(depth[i] >= 0 && depth[i] <= m.depth_limit, "node depth out of range");
        for (int d = 0; d < 3; ++d)
            MW_ARG(trans[3 * i + d] >= 0 && trans[3 * i + d] < ((long long)m.boxes[d] << depth[i]),
                   "node translation outside the world");
        key[i] = host_make_key(depth[i], trans[3 * i], trans[3 * i + 1], trans[3 * i + 2]);
        maxd = std::max(maxd, depth[i]);
    }
    // nodes already in (depth, Morton) order -- every tree this library exports -- are copied straight from
    // the caller's buffers (pinned buffers: one DMA each); otherwise the blocks are reordered on the device
    h.n = n;
    h.sorted = std::is_sorted(key.begin(), key.end());
    h.ord.resize(n);
    std::iota(h.ord.begin(), h.ord.end(), 0);
    if (!h.sorted) std::sort(h.ord.begin(), h.ord.end(), [&](int a, int b) { return key[a] < key[b]; });
    std::vector<int> pos(n);
    for (int i = 0; i < n; ++i) pos[h.ord[i]] = i;
    const int nroot = (int)((long long)m.boxes[0] * m.boxes[1] * m.boxes[2]);
    h.key.resize(n);
    h.parent.resize(n);
    h.child0.resize(n);
    h.lb.assign(maxd + 2, 0);
    int roots = 0;
    for (int i = 0; i < n; ++i) {
        const int o = h.ord[i];
        MW_ARG(parent[o] >= -1 && parent[o] < n && child0[o] >= -1 && child0[o] < n, "bad parent/child index");
        h.key[i] = key[o];
        h.parent[i] = parent[o] < 0 ? -1 : pos[parent[o]];
        h.child0[i] = child0[o] < 0 ? -1 : pos[child0[o]];
        if (depth[o] == 0) ++roots;
        h.lb[depth[o] + 1]++;
    }
    MW_ARG(roots == nroot, "tree must contain every root box");
    for (int i = 0; i < n; ++i) {
        if (h.child0[i] < 0) continue;
        const int o = h.ord[i];
        for (int c = 0; c < 8; ++c) {
            const int ch = child0[o] + c;
            MW_ARG(ch < n && pos[ch] == h.child0[i] + c && parent[ch] == o, "children must be 8 consecutive nodes");
        }
    }
    for (int d = 1; d < (int)h.lb.size(); ++d) h.lb[d] += h.lb[d - 1];
}
// Device half, in three steps on the tree's stream (nothing waits): the node arrays (through the pinned
// arena when `staged`, else direct copies that complete within the call), the coefficient blocks, then the
// hash index and norms.  upload_enqueue with a non-null coef runs all three.
static void upload_enqueue_coef(Tree& t, const HostTree& h, const double* coef) {
    Ctx* ctx = t.mra->ctx;
    cudaStream_t s = ctx->stream;
    const size_t BS = t.mra->bsize(), n = (size_t)h.n;
    if (h.sorted) {
        MWB_CUDA(cudaMemcpyAsync(t.coef, coef, sizeof(double) * BS * n, cudaMemcpyHostToDevice, s));
    } else {
        double* stage = (double*)dalloc(ctx, sizeof(double) * BS * n);
        MWB_CUDA(cudaMemcpyAsync(stage, coef, sizeof(double) * BS * n, cudaMemcpyHostToDevice, s));
        int* d_ord = (int*)dalloc(ctx, sizeof(int) * n);
        upload_bytes(ctx, d_ord, h.ord.data(), sizeof(int) * n);
        launch_gather_blocks(stage, d_ord, h.n, BS, t.coef, s);
        dfree(ctx, stage);
        dfree(ctx, d_ord);
    }
}
static void upload_enqueue_index(Tree& t, const HostTree& h) {
    cudaStream_t s = t.mra->ctx->stream;
    t.n = h.n;
    t.level_begin = h.lb;
    launch_hash_reset(t, s);
    launch_hash_insert(t, 0, h.n, s);
    launch_node_norms(t, 0, h.n, s);
}
static void upload_enqueue(Tree& t, const HostTree& h, const double* coef, bool staged) {
    Ctx* ctx = t.mra->ctx;
    cudaStream_t s = ctx->stream;
    const size_t n = (size_t)h.n;
    t.n = 0;
    tree_reserve(t, h.n);
    if (staged) {
        upload_bytes(ctx, t.key, h.key.data(), sizeof(uint64_t) * n);
        upload_bytes(ctx, t.parent, h.parent.data(), sizeof(int) * n);
        upload_bytes(ctx, t.child0, h.child0.data(), sizeof(int) * n);
    } else {
        MWB_CUDA(cudaMemcpyAsync(t.key, h.key.data(), sizeof(uint64_t) * n, cudaMemcpyHostToDevice, s));
        MWB_CUDA(cudaMemcpyAsync(t.parent, h.parent.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
        MWB_CUDA(cudaMemcpyAsync(t.child0, h.child0.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
    }
    if (coef) {
        upload_enqueue_coef(t, h, coef);
        upload_enqueue_index(t, h);
    }
}

extern "C" {

const char* mw_last_error(void) { return g_err.c_str(); }

int mw_version(int* major, int* minor) {
    MW_TRY({
        MW_ARG(major && minor, "null pointer");
        *major = 0;
        *minor = 1;
    })
}

int mw_ctx_create(int device, void* stream, mw_ctx* out) {
    MW_TRY({
        MW_ARG(out, "null pointer");
        int ndev = 0;
        MWB_CUDA(cudaGetDeviceCount(&ndev));
        MW_ARG(device >= 0 && device < ndev, "invalid CUDA device");
        MWB_CUDA(cudaSetDevice(device));
        auto* c = new mw_ctx_s();
        c->device = device;
        if (stream) {
            c->stream = (cudaStream_t)stream;
        } else {
            MWB_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
            c->own_stream = true;
        }
        MWB_CUDA(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device));
        cudaMemPool_t pool;
        MWB_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
        uint64_t thr = ~0ull;
        MWB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
        *out = c;
    })
}

int mw_ctx_set_chunk_triples(mw_ctx ctx, int flags, int triples) {
    MW_TRY({
        MW_ARG(ctx, "null context");
        MW_ARG(flags == MW_APPLY_FP64 || flags == MW_APPLY_FP32 || flags == MW_APPLY_TF32X3 || flags == MW_APPLY_BF16X3,
               "unknown apply flags");
        MW_ARG(triples >= 1 && triples <= 4096, "triples per CTA must be in [1, 4096]");
        ctx->chunk_triples[flags] = triples;
    })
}

int mw_ctx_get_chunk_triples(mw_ctx ctx, int flags, int* triples) {
    MW_TRY({
        MW_ARG(ctx && triples, "null pointer");
        MW_ARG(flags == MW_APPLY_FP64 || flags == MW_APPLY_FP32 || flags == MW_APPLY_TF32X3 || flags == MW_APPLY_BF16X3,
               "unknown apply flags");
        *triples = ctx->chunk_triples[flags];
    })
}

int mw_ctx_reserve(mw_ctx ctx, unsigned long long bytes) {
    MW_TRY({
        MW_ARG(ctx, "null context");
        MWB_CUDA(cudaSetDevice(ctx->device));
        if (bytes > 0) {
            void* p = nullptr;
            MWB_CUDA(cudaMallocAsync(&p, (size_t)bytes, ctx->stream));
            MWB_CUDA(cudaFreeAsync(p, ctx->stream));
            MWB_CUDA(cudaStreamSynchronize(ctx->stream));
        }
    })
}

int mw_ctx_profile(mw_ctx ctx, int enable) {
    MW_TRY({
        MW_ARG(ctx, "null context");
        MWB_CUDA(cudaSetDevice(ctx->device));
        if (enable && !ctx->ev0) {
            MWB_CUDA(cudaEventCreate(&ctx->ev0));
            MWB_CUDA(cudaEventCreate(&ctx->ev1));
        }
        ctx->prof = enable != 0;
        ctx->launches = 0;
        ctx->apply_launches = 0;
        ctx->apply_ctas = 0;
        ctx->apply_ms = 0.0;
    })
}

int mw_ctx_profile_ctas(mw_ctx ctx, long long* ctas) {
    MW_TRY({
        MW_ARG(ctx && ctas, "null pointer");
        *ctas = ctx->apply_ctas;
    })
}

int mw_ctx_profile_read(mw_ctx ctx, long long* launches, long long* apply_launches, double* apply_ms) {
    MW_TRY({
        MW_ARG(ctx && launches && apply_launches && apply_ms, "null pointer");
        *launches = ctx->launches;
        *apply_launches = ctx->apply_launches;
        *apply_ms = ctx->apply_ms;
    })
}

int mw_ctx_destroy(mw_ctx ctx) {
    MW_TRY({
        if (!ctx) return MW_OK;
        MW_ARG(!ctx->closed, "context destroyed twice");
        ctx->closed = true;
        if (ctx->refs == 0) ctx_free(ctx);
    })
}

int mw_ctx_synchronize(mw_ctx ctx) {
    MW_TRY({
        MW_ARG(ctx, "null context");
        MWB_CUDA(cudaSetDevice(ctx->device));
        MWB_CUDA(cudaStreamSynchronize(ctx->stream));
    })
}

int mw_mra_create(mw_ctx ctx, int min_scale, const int* corner, const int* boxes, int basis_type, int order,
                  int max_depth, mw_mra* out) {
    MW_TRY({
        MW_ARG(ctx && corner && boxes && out, "null pointer");
        MW_ARG(basis_type == MW_BASIS_INTERPOLATING || basis_type == MW_BASIS_LEGENDRE, "invalid basis type");
        MW_ARG(order >= 3 && order <= 11, "order must be in [3, 11]");
        MW_ARG(max_depth >= 0 && max_depth <= 30, "max_depth must be in [0, 30]");
        int maxb = 1;
        for (int d = 0; d < 3; ++d) {
            MW_ARG(boxes[d] >= 1 && boxes[d] <= 4096, "boxes must be in [1, 4096]");
            maxb = std::max(maxb, boxes[d]);
        }
        MWB_CUDA(cudaSetDevice(ctx->device));
        auto* m = new mw_mra_s();
        m->ctx = ctx;
        m->n0 = min_scale;
        for (int d = 0; d < 3; ++d) {
            m->corner[d] = corner[d];
            m->boxes[d] = boxes[d];
        }
        m->max_depth = max_depth;
        int lb = 0;
        while ((1 << lb) < maxb) ++lb;
        m->depth_limit = std::min(max_depth, kKeyBits - lb);
        m->basis.init(basis_type, order);
        m->k = m->basis.k;
        m->F = two_scale_filter(m->basis);
        m->W = quadrature_matrix(m->basis);
        const int k = m->k, K2 = 2 * k;
        std::vector<double> FT(K2 * K2), PF(K2 * K2, 0.0);
        for (int a = 0; a < K2; ++a)
            for (int b = 0; b < K2; ++b) FT[a * K2 + b] = m->F[b * K2 + a];
        for (int a = 0; a < K2; ++a)
            for (int c = 0; c < 2; ++c)
                for (int q = 0; q < k; ++q) {
                    double s = 0.0;
                    for (int j = 0; j < k; ++j) s += m->F[a * K2 + c * k + j] * m->W[j * k + q];
                    PF[a * K2 + c * k + q] = s;
                }
        // MV = blkdiag(E, E) F^T, E[q][j] = phi_j(x_q): compressed block -> values at the children's
        // quadrature points (up to the scale factor 2^{3(n+1)/2}), used by the pointwise product
        std::vector<double> MV(K2 * K2, 0.0), E(k * k), ph(k);
        for (int q = 0; q < k; ++q) {
            m->basis.values(m->basis.qx[q], ph.data());
            for (int j = 0; j < k; ++j) E[q * k + j] = ph[j];
        }
        for (int c = 0; c < 2; ++c)
            for (int q = 0; q < k; ++q)
                for (int b = 0; b < K2; ++b) {
                    double v = 0.0;
                    for (int j = 0; j < k; ++j) v += E[q * k + j] * m->F[b * K2 + c * k + j];
                    MV[(c * k + q) * K2 + b] = v;
                }
        cudaStream_t s = ctx->stream;
        m->d_MV = (double*)dalloc(ctx, sizeof(double) * K2 * K2);
        MWB_CUDA(cudaMemcpyAsync(m->d_MV, MV.data(), sizeof(double) * K2 * K2, cudaMemcpyHostToDevice, s));
        m->d_F = (double*)dalloc(ctx, sizeof(double) * K2 * K2);
        m->d_FT = (double*)dalloc(ctx, sizeof(double) * K2 * K2);
        m->d_PF = (double*)dalloc(ctx, sizeof(double) * K2 * K2);
        MWB_CUDA(cudaMemcpyAsync(m->d_F, m->F.data(), sizeof(double) * K2 * K2, cudaMemcpyHostToDevice, s));
        MWB_CUDA(cudaMemcpyAsync(m->d_FT, FT.data(), sizeof(double) * K2 * K2, cudaMemcpyHostToDevice, s));
        MWB_CUDA(cudaMemcpyAsync(m->d_PF, PF.data(), sizeof(double) * K2 * K2, cudaMemcpyHostToDevice, s));
        MWB_CUDA(cudaStreamSynchronize(s));
        ctx->refs++;
        *out = m;
    })
}

int mw_mra_destroy(mw_mra m) {
    MW_TRY({
        if (!m) return MW_OK;
        MW_ARG(!m->closed, "world destroyed twice");
        m->closed = true;
        if (m->refs == 0) mra_free(m);
    })
}

int mw_mra_filter(mw_mra m, double* F) {
    MW_TRY({
        MW_ARG(m && F, "null pointer");
        std::memcpy(F, m->F.data(), sizeof(double) * m->F.size());
    })
}

int mw_mra_max_depth(mw_mra m, int* depth) {
    MW_TRY({
        MW_ARG(m && depth, "null pointer");
        *depth = m->depth_limit;
    })
}

int mw_tree_create(mw_mra m, mw_tree* out) {
    MW_TRY({
        MW_ARG(m && out, "null pointer");
        MWB_CUDA(cudaSetDevice(m->ctx->device));
        auto* t = new mw_tree_s();
        t->mra = m;
        m->refs++;
        *out = t;
    })
}

int mw_tree_destroy(mw_tree t) {
    MW_TRY({
        if (!t) return MW_OK;
        Mra* m = t->mra;
        delete t;
        if (m) mra_release(m);
    })
}

int mw_tree_nnodes(mw_tree t, int* n) {
    MW_TRY({
        MW_ARG(t && n, "null pointer");
        *n = t->n;
    })
}

int mw_tree_square_norm(mw_tree t, double* out) {
    MW_TRY({
        MW_ARG(t && out, "null pointer");
        MWB_CUDA(cudaSetDevice(t->mra->ctx->device));
        *out = t->n ? reduce_leaf_norm2(*t, t->mra->ctx->stream) : 0.0;
    })
}

int mw_tree_upload(mw_tree t, int n, const int* depth, const long long* trans, const int* parent, const int* child0,
                   const double* coef) {
    MW_TRY({
        MW_ARG(t && depth && trans && parent && child0 && coef, "null pointer");
        MW_ARG(n > 0, "empty tree");
        const Mra& m = *t->mra;
        MWB_CUDA(cudaSetDevice(m.ctx->device));
        HostTree h;
        upload_prepare(m, n, depth, trans, parent, child0, h);
        upload_enqueue(*t, h, coef, false);
        MWB_CUDA(cudaStreamSynchronize(m.ctx->stream));
    })
}

int mw_tree_upload_many(int ntrees, mw_tree* trees, const int* n, const int* const* depth, const long long* const* trans,
                        const int* const* parent, const int* const* child0, const double* const* coef) {
    MW_TRY({
        MW_ARG(ntrees >= 0 && (ntrees == 0 || (trees && n && depth && trans && parent && child0 && coef)),
               "null pointer");
        std::vector<HostTree> h(ntrees);
        std::vector<cudaStream_t> streams;
        for (int i = 0; i < ntrees; ++i) {  // every check before any copy is queued
            MW_ARG(trees[i] && depth[i] && trans[i] && parent[i] && child0[i] && coef[i], "null pointer");
            MW_ARG(n[i] > 0, "empty tree");
            for (int j = 0; j < i; ++j) MW_ARG(trees[j] != trees[i], "a tree appears twice in the batch");
            MW_ARG(trees[i]->mra->ctx->device == trees[0]->mra->ctx->device, "trees on different devices");
            upload_prepare(*trees[i]->mra, n[i], depth[i], trans[i], parent[i], child0[i], h[i]);
            const cudaStream_t s = trees[i]->mra->ctx->stream;
            if (std::find(streams.begin(), streams.end(), s) == streams.end()) streams.push_back(s);
        }
        if (ntrees == 0) return MW_OK;
        MWB_CUDA(cudaSetDevice(trees[0]->mra->ctx->device));
        // node arrays first (small copies from the pinned arena), then the coefficient blocks of all trees back
        // to back, then the hash indices and norms: the copy engine streams the batch without gaps
        for (int i = 0; i < ntrees; ++i) upload_enqueue(*trees[i], h[i], nullptr, true);
        for (int i = 0; i < ntrees; ++i) upload_enqueue_coef(*trees[i], h[i], coef[i]);
        for (int i = 0; i < ntrees; ++i) upload_enqueue_index(*trees[i], h[i]);
        for (cudaStream_t s : streams) MWB_CUDA(cudaStreamSynchronize(s));
    })
}

int mw_tree_assign(mw_tree dst, mw_tree src) {
    MW_TRY({
        MW_ARG(dst && src, "null tree");
        MW_ARG(dst != src, "a tree cannot be assigned to itself");
        const Mra& a = *dst->mra;
        const Mra& b = *src->mra;
        bool same = a.ctx->device == b.ctx->device && a.k == b.k && a.basis.type == b.basis.type && a.n0 == b.n0 &&
                    a.max_depth == b.max_depth;
        for (int d = 0; d < 3; ++d) same = same && a.corner[d] == b.corner[d] && a.boxes[d] == b.boxes[d];
        MW_ARG(same, "trees on worlds with different parameters or devices");
        MWB_CUDA(cudaSetDevice(a.ctx->device));
        MWB_CUDA(cudaStreamSynchronize(b.ctx->stream));  // src complete before it is read on dst's stream
        cudaStream_t s = a.ctx->stream;
        dst->n = 0;
        tree_reserve(*dst, src->n);
        const size_t n = (size_t)src->n, BS = a.bsize();
        if (n > 0) {  // one copy kernel on dst's stream (the DMA engines may be busy with host transfers)
            mwb::CopyList L{};
            const void* from[6] = {src->key, src->parent, src->child0, src->coef, src->norm2, src->wnorm2};
            void* to[6] = {dst->key, dst->parent, dst->child0, dst->coef, dst->norm2, dst->wnorm2};
            const size_t bytes[6] = {sizeof(uint64_t) * n, sizeof(int) * n, sizeof(int) * n, sizeof(double) * BS * n,
                                     sizeof(double) * n, sizeof(double) * n};
            for (int q = 0; q < 6; ++q) {
                L.src[q] = reinterpret_cast<const unsigned char*>(from[q]);
                L.dst[q] = reinterpret_cast<unsigned char*>(to[q]);
                L.n[q] = bytes[q];
            }
            L.count = 6;
            mwb::launch_copies(a.ctx, L);
        }
        dst->n = src->n;
        dst->level_begin = src->level_begin;
        dst->g0 = src->g0;
        dst->prec = src->prec;
        for (int q = 0; q < 8; ++q) dst->stats[q] = src->stats[q];
        launch_hash_reset(*dst, s);
        launch_hash_insert(*dst, 0, dst->n, s);
        MWB_CUDA(cudaStreamSynchronize(s));  // src may change as soon as this returns
    })
}

int mw_tree_download(mw_tree t, int* depth, long long* trans, int* parent, int* child0, double* coef) {
    MW_TRY({
        MW_ARG(t, "null tree");
        const int n = t->n;
        if (n == 0) return MW_OK;
        MWB_CUDA(cudaSetDevice(t->mra->ctx->device));
        cudaStream_t s = t->mra->ctx->stream;
        std::vector<uint64_t> key(n);
        MWB_CUDA(cudaMemcpyAsync(key.data(), t->key, sizeof(uint64_t) * n, cudaMemcpyDeviceToHost, s));
        if (parent) MWB_CUDA(cudaMemcpyAsync(parent, t->parent, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
        if (child0) MWB_CUDA(cudaMemcpyAsync(child0, t->child0, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
        if (coef)
            MWB_CUDA(cudaMemcpyAsync(coef, t->coef, sizeof(double) * n * t->mra->bsize(), cudaMemcpyDeviceToHost, s));
        MWB_CUDA(cudaStreamSynchronize(s));
        for (int i = 0; i < n; ++i) {
            long long tr[3];
            host_key_trans(key[i], tr);
            if (depth) depth[i] = (int)(key[i] >> 59);
            if (trans)
                for (int d = 0; d < 3; ++d) trans[3 * i + d] = tr[d];
        }
    })
}

int mw_tree_download_many(int ntrees, mw_tree* trees, int* const* depth, long long* const* trans, int* const* parent,
                          int* const* child0, double* const* coef) {
    MW_TRY({
        MW_ARG(ntrees >= 0 && (ntrees == 0 || (trees && depth && trans && parent && child0 && coef)), "null pointer");
        std::vector<cudaStream_t> streams;
        for (int i = 0; i < ntrees; ++i) {
            MW_ARG(trees[i], "null tree");
            MW_ARG(trees[i]->mra->ctx->device == trees[0]->mra->ctx->device, "trees on different devices");
            for (int j = 0; j < i; ++j) MW_ARG(trees[j] != trees[i], "a tree appears twice in the batch");
            const cudaStream_t s = trees[i]->mra->ctx->stream;
            if (std::find(streams.begin(), streams.end(), s) == streams.end()) streams.push_back(s);
        }
        if (ntrees == 0) return MW_OK;
        MWB_CUDA(cudaSetDevice(trees[0]->mra->ctx->device));
        // keys land in the caller's trans buffer (n 8-byte words of its 3n) and are expanded in place once
        // the copies are done; without a trans buffer in a host vector
        std::vector<std::vector<uint64_t>> spare(ntrees);
        for (int i = 0; i < ntrees; ++i) {
            Tree& t = *trees[i];
            const int nn = t.n;
            if (nn == 0) continue;
            cudaStream_t s = t.mra->ctx->stream;
            void* kdst = trans[i];
            if (!kdst) {
                spare[i].resize(nn);
                kdst = spare[i].data();
            }
            MWB_CUDA(cudaMemcpyAsync(kdst, t.key, sizeof(uint64_t) * nn, cudaMemcpyDeviceToHost, s));
            if (parent[i]) MWB_CUDA(cudaMemcpyAsync(parent[i], t.parent, sizeof(int) * nn, cudaMemcpyDeviceToHost, s));
            if (child0[i]) MWB_CUDA(cudaMemcpyAsync(child0[i], t.child0, sizeof(int) * nn, cudaMemcpyDeviceToHost, s));
        }
        for (int i = 0; i < ntrees; ++i) {  // the blocks of all trees back to back
            Tree& t = *trees[i];
            if (t.n > 0 && coef[i])
                MWB_CUDA(cudaMemcpyAsync(coef[i], t.coef, sizeof(double) * t.n * t.mra->bsize(), cudaMemcpyDeviceToHost,
                                         t.mra->ctx->stream));
        }
        for (cudaStream_t s : streams) MWB_CUDA(cudaStreamSynchronize(s));
        for (int i = 0; i < ntrees; ++i) {
            const int nn = trees[i]->n;
            const unsigned char* kb =
                trans[i] ? reinterpret_cast<const unsigned char*>(trans[i]) : reinterpret_cast<const unsigned char*>(spare[i].data());
            for (int q = nn - 1; q >= 0; --q) {  // trans[3q ..] lies at or above key q: read before written
                uint64_t k;
                std::memcpy(&k, kb + sizeof(uint64_t) * q, sizeof(k));
                long long tr[3];
                host_key_trans(k, tr);
                if (depth[i]) depth[i][q] = (int)(k >> 59);
                if (trans[i])
                    for (int d = 0; d < 3; ++d) trans[i][3 * q + d] = tr[d];
            }
        }
    })
}

int mw_tree_device_arrays(mw_tree t, void** coef, void** key, void** norm2) {
    MW_TRY({
        MW_ARG(t, "null tree");
        if (coef) *coef = t->coef;
        if (key) *key = t->key;
        if (norm2) *norm2 = t->norm2;
    })
}

int mw_tree_rescale(mw_tree t, double c) {
    MW_TRY({
        MW_ARG(t, "null tree");
        MWB_CUDA(cudaSetDevice(t->mra->ctx->device));
        launch_rescale(*t, c, t->mra->ctx->stream);
        MWB_CUDA(cudaStreamSynchronize(t->mra->ctx->stream));
    })
}

int mw_project(double prec, mw_tree t, int func_type, int nparams, const double* params) {
    MW_TRY({
        MW_ARG(t && params, "null pointer");
        MWB_CUDA(cudaSetDevice(t->mra->ctx->device));
        project(prec, *t, func_type, nparams, params);
    })
}

int mw_dot(mw_tree a, mw_tree b, double* out) {
    MW_TRY({
        MW_ARG(a && b && out, "null pointer");
        MW_ARG(a->mra == b->mra, "trees must share the world");
        MWB_CUDA(cudaSetDevice(a->mra->ctx->device));
        *out = launch_dot(*a, *b, a->mra->ctx->stream);
    })
}

int mw_tree_distance(mw_tree a, mw_tree b, double* out) {
    MW_TRY({
        MW_ARG(a && b && out, "null pointer");
        MW_ARG(a->mra == b->mra, "trees on different worlds");
        MWB_CUDA(cudaSetDevice(a->mra->ctx->device));
        *out = launch_distance(*a, *b, a->mra->ctx->stream);
    })
}

int mw_op_create_poisson(mw_mra m, double prec, mw_op* out) {
    MW_TRY({
        MW_ARG(m && out, "null pointer");
        MWB_CUDA(cudaSetDevice(m->ctx->device));
        auto* op = new mw_op_s();
        try {
            op_init(*op, m, 0.0, prec);
        } catch (...) {
            delete op;
            throw;
        }
        m->refs++;
        *out = op;
    })
}

int mw_op_create_helmholtz(mw_mra m, double mu, double prec, mw_op* out) {
    MW_TRY({
        MW_ARG(m && out, "null pointer");
        MW_ARG(mu > 0.0, "mu must be positive");
        MWB_CUDA(cudaSetDevice(m->ctx->device));
        auto* op = new mw_op_s();
        try {
            op_init(*op, m, mu, prec);
        } catch (...) {
            delete op;
            throw;
        }
        m->refs++;
        *out = op;
    })
}

int mw_op_create_abgv(mw_mra m, double a, double b, mw_op* out) {
    MW_TRY({
        MW_ARG(m && out, "null pointer");
        MW_ARG(a >= 0.0 && a <= 1.0 && b >= 0.0 && b <= 1.0, "flux parameters must lie in [0, 1]");
        MWB_CUDA(cudaSetDevice(m->ctx->device));
        auto* op = new mw_op_s();
        op->mra = m;
        op->kind = 1;
        op->da = a;
        op->db = b;
        derivative_blocks(m->basis, a, b, op->dT);
        m->refs++;
        *out = op;
    })
}

int mw_apply_derivative(mw_tree out, mw_op op, mw_tree inp, int dir, int flags) {
    MW_TRY({
        MW_ARG(out && op && inp, "null pointer");
        MW_ARG(flags == MW_APPLY_FP64 || flags == MW_APPLY_FP32 || flags == MW_APPLY_TF32X3 || flags == MW_APPLY_BF16X3,
               "unknown apply flags");
        MWB_CUDA(cudaSetDevice(inp->mra->ctx->device));
        apply_derivative(out, op, inp, dir, flags);
    })
}

int mw_op_destroy(mw_op op) {
    MW_TRY({
        if (!op) return MW_OK;
        Mra* m = op->mra;
        delete op;
        if (m) mra_release(m);
    })
}

int mw_op_nterms(mw_op op, int* n) {
    MW_TRY({
        MW_ARG(op && n, "null pointer");
        *n = (int)op->terms.size();
    })
}

int mw_op_terms(mw_op op, double* alpha, double* beta) {
    MW_TRY({
        MW_ARG(op && alpha && beta, "null pointer");
        for (size_t i = 0; i < op->terms.size(); ++i) {
            alpha[i] = op->terms[i].alpha;
            beta[i] = op->terms[i].beta;
        }
    })
}

int mw_op_scaling_matrix(mw_op op, double alpha, int n, long long l, double* T) {
    MW_TRY({
        MW_ARG(op && T, "null pointer");
        MW_ARG(op->kind == 0 && op->builder, "not a separated-Gaussian convolution operator");
        MW_ARG(alpha > 0.0, "alpha must be positive");
        op->builder->scaling(alpha, n, (long)l, T);
    })
}

int mw_op_ns_matrix(mw_op op, int term, int n, long long l, double* NS) {
    MW_TRY({
        MW_ARG(op && NS, "null pointer");
        MW_ARG(op->kind == 0 && op->builder, "not a separated-Gaussian convolution operator");
        MW_ARG(term >= 0 && term < (int)op->terms.size(), "term index out of range");
        std::vector<std::pair<long, std::vector<double>>> cache;
        op->builder->ns(op->terms[term].alpha, n, (long)l, NS, cache);
    })
}

int mw_apply(double prec, mw_tree out, mw_op op, mw_tree inp, int flags) {
    MW_TRY({
        MW_ARG(out && op && inp, "null pointer");
        MW_ARG(flags == MW_APPLY_FP64 || flags == MW_APPLY_FP32 || flags == MW_APPLY_TF32X3 || flags == MW_APPLY_BF16X3,
               "unknown apply flags");
        MWB_CUDA(cudaSetDevice(inp->mra->ctx->device));
        Tree* o = out;
        Op* p = op;
        Tree* i = inp;
        apply_batched(prec, 1, &o, &p, &i, flags);
    })
}

int mw_apply_batched(int n, double prec, mw_tree* out, mw_op* ops, mw_tree* inp, int flags) {
    MW_TRY({
        MW_ARG(n > 0 && out && ops && inp, "null pointer or empty batch");
        MW_ARG(flags == MW_APPLY_FP64 || flags == MW_APPLY_FP32 || flags == MW_APPLY_TF32X3 || flags == MW_APPLY_BF16X3,
               "unknown apply flags");
        MW_ARG(inp[0], "null input tree");
        MWB_CUDA(cudaSetDevice(inp[0]->mra->ctx->device));
        std::vector<Tree*> o(n), i(n);
        std::vector<Op*> p(n);
        for (int q = 0; q < n; ++q) {
            o[q] = out[q];
            p[q] = ops[q];
            i[q] = inp[q];
        }
        apply_batched(prec, n, o.data(), p.data(), i.data(), flags);
    })
}

int mw_apply_stats(mw_tree out, long long* stats) {
    MW_TRY({
        MW_ARG(out && stats, "null pointer");
        for (int i = 0; i < 4; ++i) stats[i] = out->stats[i];
    })
}

int mw_mlp_create(mw_ctx ctx, int hidden_layers, int width, unsigned seed, mw_mlp* out) {
    MW_TRY({
        MW_ARG(ctx && out, "null pointer");
        MW_ARG(hidden_layers >= 1 && hidden_layers <= 8 && width >= 8 && width <= 512, "bad network shape");
        MWB_CUDA(cudaSetDevice(ctx->device));
        auto* M = new mw_mlp_s();
        mlp_init(*M, ctx, hidden_layers, width, seed);
        ctx->refs++;
        *out = M;
    })
}

int mw_mlp_destroy(mw_mlp mlp) {
    MW_TRY({
        if (!mlp) return MW_OK;
        Ctx* c = mlp->ctx;
        delete mlp;
        if (c) ctx_release(c);
    })
}

int mw_mlp_nparams(mw_mlp mlp, long long* n, int* nfeatures) {
    MW_TRY({
        MW_ARG(mlp && n && nfeatures, "null pointer");
        *n = (long long)mlp->nparam;
        *nfeatures = kNF;
    })
}

int mw_mlp_get_params(mw_mlp mlp, float* p) {
    MW_TRY({
        MW_ARG(mlp && p, "null pointer");
        MWB_CUDA(cudaSetDevice(mlp->ctx->device));
        MWB_CUDA(cudaMemcpyAsync(p, mlp->d_p, sizeof(float) * mlp->nparam, cudaMemcpyDeviceToHost, mlp->ctx->stream));
        MWB_CUDA(cudaStreamSynchronize(mlp->ctx->stream));
    })
}

int mw_mlp_set_params(mw_mlp mlp, const float* p) {
    MW_TRY({
        MW_ARG(mlp && p, "null pointer");
        MWB_CUDA(cudaSetDevice(mlp->ctx->device));
        MWB_CUDA(cudaMemcpyAsync(mlp->d_p, p, sizeof(float) * mlp->nparam, cudaMemcpyHostToDevice, mlp->ctx->stream));
        MWB_CUDA(cudaStreamSynchronize(mlp->ctx->stream));
    })
}

int mw_mlp_forward(mw_mlp mlp, int n, const float* x, float* logits) {
    MW_TRY({
        MW_ARG(mlp && x && logits && n > 0, "null pointer or empty input");
        Ctx* ctx = mlp->ctx;
        MWB_CUDA(cudaSetDevice(ctx->device));
        float* d_X = (float*)dalloc(ctx, sizeof(float) * (size_t)n * kNF);
        MWB_CUDA(cudaMemcpyAsync(d_X, x, sizeof(float) * (size_t)n * kNF, cudaMemcpyHostToDevice, ctx->stream));
        std::vector<float> z = mlp_logits(*mlp, d_X, n, ctx->stream);
        std::copy(z.begin(), z.end(), logits);
        dfree(ctx, d_X);
        MWB_CUDA(cudaStreamSynchronize(ctx->stream));
    })
}

int mw_mlp_gradient(mw_mlp mlp, int n, const float* x, const float* y, const float* w, double* loss, float* grad) {
    MW_TRY({
        MW_ARG(mlp && x && y && w && loss && grad && n > 0, "null pointer or empty input");
        Ctx* ctx = mlp->ctx;
        cudaStream_t s = ctx->stream;
        MWB_CUDA(cudaSetDevice(ctx->device));
        float* d_X = (float*)dalloc(ctx, sizeof(float) * (size_t)n * kNF);
        float* d_y = (float*)dalloc(ctx, sizeof(float) * n);
        float* d_w = (float*)dalloc(ctx, sizeof(float) * n);
        MWB_CUDA(cudaMemcpyAsync(d_X, x, sizeof(float) * (size_t)n * kNF, cudaMemcpyHostToDevice, s));
        MWB_CUDA(cudaMemcpyAsync(d_y, y, sizeof(float) * n, cudaMemcpyHostToDevice, s));
        MWB_CUDA(cudaMemcpyAsync(d_w, w, sizeof(float) * n, cudaMemcpyHostToDevice, s));
        std::vector<float*> acts;
        mlp_forward(*mlp, d_X, n, acts, s);
        *loss = mlp_backward(*mlp, acts, d_y, d_w, n, s);
        free_acts(*mlp, acts);
        MWB_CUDA(cudaMemcpyAsync(grad, mlp->d_g, sizeof(float) * mlp->nparam, cudaMemcpyDeviceToHost, s));
        MWB_CUDA(cudaStreamSynchronize(s));
        for (float* q : {d_X, d_y, d_w}) dfree(ctx, q);
    })
}

int mw_mlp_collect(mw_mlp mlp, mw_tree out, mw_op op, mw_tree inp) {
    MW_TRY({
        MW_ARG(mlp && out && op && inp, "null pointer");
        MW_ARG(out->g0 > 0.0 && out->prec > 0.0, "output tree has no apply to learn from");
        MWB_CUDA(cudaSetDevice(mlp->ctx->device));
        collect_training(*mlp, *out, *op, *inp);
    })
}

int mw_mlp_dataset(mw_mlp mlp, int* n, int* npos) {
    MW_TRY({
        MW_ARG(mlp && n && npos, "null pointer");
        *n = mlp->n_data;
        std::vector<float> y(mlp->n_data);
        if (mlp->n_data) {
            MWB_CUDA(cudaMemcpyAsync(y.data(), mlp->d_y, sizeof(float) * y.size(), cudaMemcpyDeviceToHost, mlp->ctx->stream));
            MWB_CUDA(cudaStreamSynchronize(mlp->ctx->stream));
        }
        int p = 0;
        for (float v : y) p += v > 0.5f;
        *npos = p;
    })
}

int mw_mlp_dataset_get(mw_mlp mlp, float* x, float* y) {
    MW_TRY({
        MW_ARG(mlp && x && y, "null pointer");
        cudaStream_t s = mlp->ctx->stream;
        MWB_CUDA(cudaMemcpyAsync(x, mlp->d_X, sizeof(float) * (size_t)mlp->n_data * kNF, cudaMemcpyDeviceToHost, s));
        MWB_CUDA(cudaMemcpyAsync(y, mlp->d_y, sizeof(float) * mlp->n_data, cudaMemcpyDeviceToHost, s));
        MWB_CUDA(cudaStreamSynchronize(s));
    })
}

int mw_mlp_train(mw_mlp mlp, int epochs, int batch, float lr, unsigned seed, double* loss) {
    MW_TRY({
        MW_ARG(mlp && loss && epochs > 0 && batch > 0 && lr > 0.0f, "bad training arguments");
        MWB_CUDA(cudaSetDevice(mlp->ctx->device));
        *loss = mlp_train(*mlp, epochs, batch, lr, seed);
    })
}

int mw_apply_learned(int n, double prec, mw_tree* out, mw_op* ops, mw_tree* inp, int flags, mw_mlp mlp, float tau,
                     long long* stats) {
    MW_TRY({
        MW_ARG(n > 0 && out && ops && inp && mlp, "null pointer or empty batch");
        MW_ARG(flags == MW_APPLY_FP64 || flags == MW_APPLY_FP32 || flags == MW_APPLY_TF32X3 || flags == MW_APPLY_BF16X3,
               "unknown apply flags");
        MW_ARG(tau > 0.0f && tau < 1.0f, "tau must be in (0, 1)");
        MW_ARG(inp[0], "null input tree");
        MW_ARG(mlp->ctx == inp[0]->mra->ctx, "the network and the trees belong to different contexts");
        MWB_CUDA(cudaSetDevice(inp[0]->mra->ctx->device));
        std::vector<Tree*> o(n), i(n);
        std::vector<Op*> p(n);
        for (int q = 0; q < n; ++q) {
            o[q] = out[q];
            p[q] = ops[q];
            i[q] = inp[q];
        }
        apply_learned(prec, n, o.data(), p.data(), i.data(), flags, *mlp, tau, stats);
    })
}

}  // extern "C"
