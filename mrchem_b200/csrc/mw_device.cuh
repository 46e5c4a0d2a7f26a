// mw_device.cuh -- device helpers shared by the kernels: Morton node keys, the open-addressing hash
// index, block geometry of a node, block reductions and the in-place pencil transform.
#pragma once
#include <cstdint>

#include "mw_internal.hpp"

namespace mwb {

// ---------------------------------------------------------------------------------------------
// keys and hash index
// ---------------------------------------------------------------------------------------------

__host__ __device__ static inline uint64_t spread3(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | v << 32) & 0x1f00000000ffffull;
    v = (v | v << 16) & 0x1f0000ff0000ffull;
    v = (v | v << 8) & 0x100f00f00f00f00full;
    v = (v | v << 4) & 0x10c30c30c30c30c3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
}
__host__ __device__ static inline uint64_t compact3(uint64_t v) {
    v &= 0x1249249249249249ull;
    v = (v ^ (v >> 2)) & 0x10c30c30c30c30c3ull;
    v = (v ^ (v >> 4)) & 0x100f00f00f00f00full;
    v = (v ^ (v >> 8)) & 0x1f0000ff0000ffull;
    v = (v ^ (v >> 16)) & 0x1f00000000ffffull;
    v = (v ^ (v >> 32)) & 0x1fffffull;
    return v;
}
__host__ __device__ static inline uint64_t make_key(int depth, long long tx, long long ty, long long tz) {
    return ((uint64_t)depth << 59) | spread3((uint64_t)tx) | (spread3((uint64_t)ty) << 1) |
           (spread3((uint64_t)tz) << 2);
}
__host__ __device__ static inline int key_depth(uint64_t k) { return (int)(k >> 59); }
__host__ __device__ static inline void key_trans(uint64_t k, long long t[3]) {
    uint64_t m = k & ((1ull << 57) - 1);
    t[0] = (long long)compact3(m);
    t[1] = (long long)compact3(m >> 1);
    t[2] = (long long)compact3(m >> 2);
}
__device__ static inline uint32_t hslot(uint64_t k, uint32_t mask) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return (uint32_t)k & mask;
}
// linear probing; at most `cap` probes (the table is kept at most half full)
__device__ static inline int hlookup(const uint64_t* hk, const int* hv, uint32_t cap, uint64_t key) {
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

// 16-byte asynchronous global -> shared copies (cp.async, L2 only), their commit and completion
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(smem_dst)),
                 "l"(gmem_src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// wait until at most N of this thread's most recently committed groups are pending
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
// prefetch the 16-byte-aligned part of [gmem, gmem + bytes) into L2 through the bulk-copy engine
// (the instruction wants a 16-byte aligned address and a size that is a multiple of 16)
__device__ __forceinline__ void prefetch_l2_bulk(const void* gmem, unsigned bytes) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(gmem);
    const uintptr_t lo = (a + 15) & ~uintptr_t(15), hi = (a + bytes) & ~uintptr_t(15);
    if (hi > lo)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(lo), "r"((unsigned)(hi - lo)) : "memory");
}

// Sum two values over the block; the result is valid in thread 0.  `red` holds 64 doubles.
__device__ static inline void block_sum2(double& a, double& b, double* red) {
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
__device__ static inline void pencil_transform(const double* __restrict__ M, double* A) {
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

}  // namespace mwb
