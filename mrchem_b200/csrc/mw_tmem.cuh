// Tensor memory (TMEM) as per-thread accumulator storage on sm_100a.
//
// The contraction kernel keeps each output node's FP64 accumulators for the whole chunk of
// (input node, term) pairs.  In the mixed-precision kernel they do not fit in registers next to the
// FP32 GEMM tiles, so they live in TMEM: 128 lanes x 512 columns of 32-bit cells per SM.  A warp may
// touch only its lane quarter (lanes 32 (warp % 4) ...); with the 32x32b shape thread t of the warp
// reads and writes its own lane, N consecutive columns per instruction.  A double occupies two
// consecutive columns (low word first).
//
// Protocol used here (PTX ISA, tcgen05 family):
//   - one warp allocates (power-of-two column count >= 32), writes the address to shared memory and
//     gives up the allocation permit; all threads read it after a fenced barrier;
//   - loads complete at tcgen05.wait::ld, which takes the destination registers as operands so that
//     no use of them can be scheduled before it; stores are waited for with tcgen05.wait::st before
//     the same cells are loaded again;
//   - before the allocating warp frees the columns every warp's accesses are ordered by a fenced
//     barrier.
#pragma once
#include <cstdint>

namespace mwb {

__device__ __forceinline__ uint32_t smem_addr_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr_u32(slot)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tmem_fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// 32x32b loads / stores of N = 2, 4, 8, 16 consecutive columns
template <int N> struct Tmem;

template <> struct Tmem<2> {
    __device__ static __forceinline__ void ld(uint32_t a, uint32_t (&r)[2]) {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(r[0]), "=r"(r[1]) : "r"(a) : "memory");
    }
    __device__ static __forceinline__ void wait(uint32_t (&r)[2]) {
        asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(r[0]), "+r"(r[1])::"memory");
    }
    __device__ static __forceinline__ void st(uint32_t a, const uint32_t (&r)[2]) {
        asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(a), "r"(r[0]), "r"(r[1]) : "memory");
    }
};

template <> struct Tmem<4> {
    __device__ static __forceinline__ void ld(uint32_t a, uint32_t (&r)[4]) {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                     : "r"(a)
                     : "memory");
    }
    __device__ static __forceinline__ void wait(uint32_t (&r)[4]) {
        asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3])::"memory");
    }
    __device__ static __forceinline__ void st(uint32_t a, const uint32_t (&r)[4]) {
        asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(a), "r"(r[0]), "r"(r[1]),
                     "r"(r[2]), "r"(r[3])
                     : "memory");
    }
};

template <> struct Tmem<8> {
    __device__ static __forceinline__ void ld(uint32_t a, uint32_t (&r)[8]) {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                     : "r"(a)
                     : "memory");
    }
    __device__ static __forceinline__ void wait(uint32_t (&r)[8]) {
        asm volatile("tcgen05.wait::ld.sync.aligned;"
                     : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7])::"memory");
    }
    __device__ static __forceinline__ void st(uint32_t a, const uint32_t (&r)[8]) {
        asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(a), "r"(r[0]),
                     "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
                     : "memory");
    }
};

template <> struct Tmem<16> {
    __device__ static __forceinline__ void ld(uint32_t a, uint32_t (&r)[16]) {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
            "%15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
              "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(a)
            : "memory");
    }
    __device__ static __forceinline__ void wait(uint32_t (&r)[16]) {
        asm volatile("tcgen05.wait::ld.sync.aligned;"
                     : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                       "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                       "+r"(r[15])::"memory");
    }
    __device__ static __forceinline__ void st(uint32_t a, const uint32_t (&r)[16]) {
        asm volatile(
            "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
            "%15, %16};" ::"r"(a),
            "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
            "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
            : "memory");
    }
};

__device__ __forceinline__ double words_to_double(uint32_t lo, uint32_t hi) {
    return __hiloint2double(static_cast<int>(hi), static_cast<int>(lo));
}
__device__ __forceinline__ void double_to_words(double v, uint32_t& lo, uint32_t& hi) {
    lo = static_cast<uint32_t>(__double2loint(v));
    hi = static_cast<uint32_t>(__double2hiint(v));
}

// Visit the ND doubles of a thread's TMEM accumulator block in groups (8, then 4, 2, 1):
// f(first_double, group_doubles, words) may read and modify the words; modified groups are stored back
// when `write` is set.  Every lane of the warp must call this (the TMEM accesses are warp-collective).
template <int ND, bool WRITE, typename F>
__device__ __forceinline__ void tmem_visit(uint32_t taddr, F&& f) {
    constexpr int N8 = ND / 8;
#pragma unroll
    for (int g = 0; g < N8; ++g) {
        uint32_t r[16];
        Tmem<16>::ld(taddr + 16 * g, r);
        Tmem<16>::wait(r);
        f(8 * g, 8, r);
        if (WRITE) Tmem<16>::st(taddr + 16 * g, r);
    }
    constexpr int rem = ND - 8 * N8;
    int d0 = 8 * N8;
    if constexpr ((rem & 4) != 0) {
        uint32_t r[8];
        Tmem<8>::ld(taddr + 2 * d0, r);
        Tmem<8>::wait(r);
        f(d0, 4, r);
        if (WRITE) Tmem<8>::st(taddr + 2 * d0, r);
        d0 += 4;
    }
    if constexpr ((rem & 2) != 0) {
        uint32_t r[4];
        Tmem<4>::ld(taddr + 2 * d0, r);
        Tmem<4>::wait(r);
        f(d0, 2, r);
        if (WRITE) Tmem<4>::st(taddr + 2 * d0, r);
        d0 += 2;
    }
    if constexpr ((rem & 1) != 0) {
        uint32_t r[2];
        Tmem<2>::ld(taddr + 2 * d0, r);
        Tmem<2>::wait(r);
        f(d0, 1, r);
        if (WRITE) Tmem<2>::st(taddr + 2 * d0, r);
    }
    if (WRITE) tmem_wait_st();
}

}  // namespace mwb
