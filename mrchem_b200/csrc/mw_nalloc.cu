// mw_nalloc.cu -- inner product of two trees that allocates no device memory.
//
// Why it exists: some callers cannot allocate device memory at the moment they need a result -- code
// running under a fixed memory budget that pre-reserves everything at start-up, a caller that has
// handed the whole device memory pool to another framework, or a thread that must not touch the
// allocator while other work is being recorded on its device.  mw_dot() allocates two small scratch
// buffers from the stream-ordered pool on every call; mw_nalloc_dot() computes the same sum with its
// scratch in a fixed, file-scope device array instead.  The call itself ends with a blocking read of
// the result into host memory, so it is not a call to place inside a CUDA graph capture.
//
// The array g_nalloc_scratch holds kNallocMaxNodes per-node partial sums plus one slot for the
// total (8 MiB + 256 B).  Every GPU that loads this library holds it until the process exits.  Its
// device address is looked up once per device with cudaGetSymbolAddress (the symbol name itself is
// only a host-side stand-in and must never be passed to a kernel).
#include <mutex>
#include <string>

#include "../../include/mwb200.h"
#include "mw_device.cuh"
#include "mw_internal.hpp"

namespace mwb {
void set_last_error(const std::string& msg);
}

namespace {

constexpr int kNallocMaxNodes = 1 << 20;  // largest tree (node count) the allocation-free dot accepts
constexpr int kNallocSlots = kNallocMaxNodes + 32;

// [0, kNallocMaxNodes): per-node partial sums of the current call; [kNallocMaxNodes]: the total
static __device__ __align__(256) double g_nalloc_scratch[kNallocSlots];

std::mutex g_nalloc_mtx;
double* g_nalloc_ptr[256] = {};  // device address of g_nalloc_scratch, per CUDA device

// Device address of the scratch array on `device`, which must be the current device.  Looked up on
// the first call per device; that first call must therefore not happen while the calling thread is
// capturing a CUDA graph.
double* nalloc_scratch(int device) {
    std::lock_guard<std::mutex> lk(g_nalloc_mtx);
    if (device < 0 || device >= 256) throw mwb::Error(MW_ERR_ARG, "device index out of range");
    if (!g_nalloc_ptr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_nalloc_scratch);
        if (e != cudaSuccess || p == nullptr)
            throw mwb::Error(MW_ERR_CUDA, std::string("cudaGetSymbolAddress(g_nalloc_scratch): ") +
                                              cudaGetErrorString(e));
        g_nalloc_ptr[device] = (double*)p;
    }
    return g_nalloc_ptr[device];
}

// one warp per node of a: <a_node|b_node> over the wavelet part (all components at the root
// depth); every partial in [0, na) is written, so no slot needs clearing between calls
__global__ void k_nalloc_dot_nodes(const uint64_t* __restrict__ akey, const double* __restrict__ acoef, int na,
                                   const double* __restrict__ bcoef, const uint64_t* hk, const int* hv,
                                   uint32_t hcap, int k, double* part) {
    const int node = (blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x & 31;
    if (node >= na) return;
    const int K2 = 2 * k, BS = K2 * K2 * K2;
    const uint64_t key = akey[node];
    const int j = mwb::hlookup(hk, hv, hcap, key);  // the trees' own hash index (mw_device.cuh)
    double s = 0.0;
    if (j >= 0) {
        const bool root = mwb::key_depth(key) == 0;
        const double* x = acoef + (size_t)node * BS;
        const double* y = bcoef + (size_t)j * BS;
        for (int e = lane; e < BS; e += 32) {
            const int a = e % K2, b = (e / K2) % K2, c = e / (K2 * K2);
            if (!root && a < k && b < k && c < k) continue;
            s += x[e] * y[e];
        }
    }
    for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) part[node] = s;
}

// fixed-order sum of part[0, n) into part[kNallocMaxNodes] (single block)
__global__ void k_nalloc_sum(double* part, int n) {
    __shared__ double red[32];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += part[i];
    for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = s;
    __syncthreads();
    if (w == 0) {
        s = l < (int)(blockDim.x >> 5) ? red[l] : 0.0;
        for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (l == 0) part[kNallocMaxNodes] = s;
    }
}

}  // namespace

struct mw_tree_s : mwb::Tree {};

extern "C" int mw_nalloc_dot(mw_tree a, mw_tree b, double* out) {
    try {
        if (!a || !b || !out) throw mwb::Error(MW_ERR_ARG, "null pointer");
        if (a->mra != b->mra) throw mwb::Error(MW_ERR_ARG, "trees must share the world");
        if (a->n > kNallocMaxNodes)
            throw mwb::Error(MW_ERR_CAPACITY, "tree has " + std::to_string(a->n) +
                                                  " nodes; mw_nalloc_dot accepts at most " +
                                                  std::to_string(kNallocMaxNodes) + " (use mw_dot)");
        if (a->n == 0 || b->n == 0) {
            *out = 0.0;
            return MW_OK;
        }
        mwb::Ctx* ctx = a->mra->ctx;
        MWB_CUDA(cudaSetDevice(ctx->device));
        double* part = nalloc_scratch(ctx->device);
        cudaStream_t s = ctx->stream;
        k_nalloc_dot_nodes<<<(a->n * 32 + 255) / 256, 256, 0, s>>>(a->key, a->coef, a->n, b->coef, b->hkey, b->hval,
                                                                   b->hcap, a->mra->k, part);
        k_nalloc_sum<<<1, 1024, 0, s>>>(part, a->n);
        MWB_CUDA(cudaGetLastError());
        MWB_CUDA(cudaMemcpyAsync(out, part + kNallocMaxNodes, sizeof(double), cudaMemcpyDeviceToHost, s));
        MWB_CUDA(cudaStreamSynchronize(s));
        return MW_OK;
    } catch (const mwb::Error& e) {
        mwb::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        mwb::set_last_error(e.what());
        return MW_ERR_STATE;
    }
}
