// mw_umma.cuh -- the fifth-generation tensor-core (tcgen05) primitives of the contraction kernel.
//
// Only the forms that the contraction uses, all checked on sm_100a by exact small-integer products:
//   - operands in shared memory without swizzling and K-major: an operand of R rows and 4-element
//     (16-byte) K chunks keeps element (r, k) at byte 16 (r + RS (k / 4)) + 4 (k % 4) from its base,
//     i.e. "core matrices" of 8 rows x 16 bytes stacked every 128 bytes along the rows and every
//     16 RS bytes along K; RS is any row count >= the rows read;
//   - kind::tf32, FP32 accumulation in tensor memory, M = 128 rows (TMEM lane = row), N a multiple
//     of 8, K = 8 per instruction (two chunks);
//   - completion through tcgen05.commit on an mbarrier, waited for with a time limit.
// The descriptor fields follow the shared-memory and instruction descriptor tables of the PTX ISA
// (tcgen05 matrix descriptors): start address, leading-dimension byte offset (the K-chunk stride here)
// and stride-dimension byte offset (the 8-row stride), all in 16-byte units, descriptor version 1,
// layout type 0 (no swizzle).  (The MN-major form of the A operand returned zeros for kind::tf32 in
// the same checks, so every operand here is K-major.)
#pragma once
#include <cstdint>
#include <utility>

#include "mw_tmem.cuh"

namespace mwb {

// ---- mbarrier -------------------------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Wait for the phase with the given parity to complete; false after `limit_ns` without completion.
// (try_wait itself suspends the thread for a while; the clock is read every 64 polls.)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
    const uint32_t a = smem_addr_u32(bar);
    uint64_t t0 = 0;
    for (uint32_t it = 0;; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if ((it & 63u) == 0) {
            const uint64_t t = global_ns();
            if (it == 0) t0 = t;
            else if (t - t0 > limit_ns) return false;
        }
    }
}

// ---- fences ---------------------------------------------------------------------------------------
// generic-proxy shared-memory writes (st.shared, cp.async) -> visible to the tensor core's reads
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ---- descriptors ----------------------------------------------------------------------------------
// K-major, no swizzle: lbo = byte stride between 16-byte K chunks, sbo = byte stride between 8-row groups
__device__ __forceinline__ uint64_t umma_sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version (sm_100)
    return d;                // base offset 0, layout type 0 (no swizzle)
}
// kind::tf32 instruction descriptor: D FP32, A and B TF32, both K-major, M x N
__host__ __device__ constexpr uint32_t umma_idesc_tf32(int m, int n) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// ---- MMA, commit ----------------------------------------------------------------------------------
// D[tmem] (+)= A B^T, one 128 x N x 8 step; issued by one thread
__device__ __forceinline__ void umma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}
// kind::f16 instruction descriptor with BF16 A and B (format 1 in both fields), FP32 D, both K-major,
// M x N (M = 128: N a multiple of 16 up to 256); one instruction contracts K = 16
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}
// D[tmem] (+)= A B^T, one 128 x N x 16 step of BF16 operands; issued by one thread
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

// ---- 1-D bulk copies (TMA engine, no tensor map, no multicast) ------------------------------------
// The thread that arms a stage announces the bytes it expects; the copies complete the transaction
// count on the same mbarrier.  Sizes are multiples of 16 bytes, both addresses 16-byte aligned.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* smem_dst, const void* gmem_src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr_u32(smem_dst)),
        "l"(gmem_src), "r"(bytes), "r"(smem_addr_u32(bar))
        : "memory");
}

// arrive on `bar` once every MMA this thread issued before has completed
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_addr_u32(bar))
                 : "memory");
}

// ---- TF32 split -----------------------------------------------------------------------------------
// FP32 -> TF32 (10 explicit mantissa bits), nearest with ties away from zero, by integer arithmetic on
// the bit pattern (the conversion unit stays free); finite inputs only
__device__ __forceinline__ uint32_t tf32_rn(float x) { return (__float_as_uint(x) + 0x1000u) & 0xffffe000u; }
// x = hi + lo + O(2^-22 |x|): hi = TF32 rounding of x, lo = TF32 rounding of the remainder
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
    hi = tf32_rn(x);
    lo = tf32_rn(x - __uint_as_float(hi));
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d) : "memory");
}

// f(std::integral_constant<int, i>) for i = 0 .. N-1, unrolled at compile time
template <typename F, int... I>
__device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, I...>) {
    (f(std::integral_constant<int, I>{}), ...);
}
template <int N, typename F>
__device__ __forceinline__ void static_for(F&& f) {
    static_for_impl(f, std::make_integer_sequence<int, N>{});
}

// N consecutive TMEM columns of this thread's lane <-> r[OFF .. OFF + N) (32x32b shape, pieces of
// 8, 4, 2, 1 columns).  tmem_span_wait must follow the loads before r is read: it binds the registers
// to the wait so that no use is scheduled ahead of it.
template <int OFF, int N, int ARR>
__device__ __forceinline__ void tmem_span_ld(uint32_t a, uint32_t (&r)[ARR]) {
    static_assert(OFF + N <= ARR, "span");
    if constexpr (N >= 8) {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                     : "=r"(r[OFF]), "=r"(r[OFF + 1]), "=r"(r[OFF + 2]), "=r"(r[OFF + 3]), "=r"(r[OFF + 4]),
                       "=r"(r[OFF + 5]), "=r"(r[OFF + 6]), "=r"(r[OFF + 7])
                     : "r"(a)
                     : "memory");
        tmem_span_ld<OFF + 8, N - 8>(a + 8, r);
    } else if constexpr (N >= 4) {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                     : "=r"(r[OFF]), "=r"(r[OFF + 1]), "=r"(r[OFF + 2]), "=r"(r[OFF + 3])
                     : "r"(a)
                     : "memory");
        tmem_span_ld<OFF + 4, N - 4>(a + 4, r);
    } else if constexpr (N >= 2) {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];"
                     : "=r"(r[OFF]), "=r"(r[OFF + 1])
                     : "r"(a)
                     : "memory");
        tmem_span_ld<OFF + 2, N - 2>(a + 2, r);
    } else if constexpr (N == 1) {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r[OFF]) : "r"(a) : "memory");
    }
}
template <int OFF, int N, int ARR>
__device__ __forceinline__ void tmem_span_wait(uint32_t (&r)[ARR]) {
    if constexpr (N >= 4) {
        asm volatile("tcgen05.wait::ld.sync.aligned;"
                     : "+r"(r[OFF]), "+r"(r[OFF + 1]), "+r"(r[OFF + 2]), "+r"(r[OFF + 3])::"memory");
        tmem_span_wait<OFF + 4, N - 4>(r);
    } else if constexpr (N >= 1) {
        asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(r[OFF])::"memory");
        tmem_span_wait<OFF + 1, N - 1>(r);
    }
}
template <int OFF, int N, int ARR>
__device__ __forceinline__ void tmem_span_st(uint32_t a, const uint32_t (&r)[ARR]) {
    static_assert(OFF + N <= ARR, "span");
    if constexpr (N >= 8) {
        asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(a),
                     "r"(r[OFF]), "r"(r[OFF + 1]), "r"(r[OFF + 2]), "r"(r[OFF + 3]), "r"(r[OFF + 4]), "r"(r[OFF + 5]),
                     "r"(r[OFF + 6]), "r"(r[OFF + 7])
                     : "memory");
        tmem_span_st<OFF + 8, N - 8>(a + 8, r);
    } else if constexpr (N >= 4) {
        asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(a), "r"(r[OFF]),
                     "r"(r[OFF + 1]), "r"(r[OFF + 2]), "r"(r[OFF + 3])
                     : "memory");
        tmem_span_st<OFF + 4, N - 4>(a + 4, r);
    } else if constexpr (N >= 2) {
        asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(a), "r"(r[OFF]), "r"(r[OFF + 1])
                     : "memory");
        tmem_span_st<OFF + 2, N - 2>(a + 2, r);
    } else if constexpr (N == 1) {
        asm volatile("tcgen05.st.sync.aligned.32x32b.x1.b32 [%0], {%1};" ::"r"(a), "r"(r[OFF]) : "memory");
    }
}

// 4 x 4 transpose inside each quad of lanes (lanes 4q .. 4q+3, j = lane % 4): on entry x[c] is column c
// of row j, on exit x[i] is column j of row i.  Every lane of the warp must take part.
__device__ __forceinline__ void quad_transpose(float (&x)[4], int j) {
    const bool h = (j & 2) != 0;
    float s0 = h ? x[0] : x[2], s1 = h ? x[1] : x[3];
    float t0 = __shfl_xor_sync(0xffffffffu, s0, 2), t1 = __shfl_xor_sync(0xffffffffu, s1, 2);
    if (h) {
        x[0] = t0;
        x[1] = t1;
    } else {
        x[2] = t0;
        x[3] = t1;
    }
    const bool l = (j & 1) != 0;
    s0 = l ? x[0] : x[1];
    s1 = l ? x[2] : x[3];
    t0 = __shfl_xor_sync(0xffffffffu, s0, 1);
    t1 = __shfl_xor_sync(0xffffffffu, s1, 1);
    if (l) {
        x[0] = t0;
        x[2] = t1;
    } else {
        x[1] = t0;
        x[3] = t1;
    }
}

}  // namespace mwb
