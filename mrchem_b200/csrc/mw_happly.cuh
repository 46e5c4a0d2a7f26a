// mw_happly.cuh -- line-ordered contraction of the NS-form apply with its x step on the fifth-generation
// tensor cores (tcgen05.mma kind::f16, BF16 operands) and its y and z steps on the CUDA cores (FP32
// products); every term's contribution is accumulated in FP64.  Included by mw_apply.cu after the Chunk /
// Item / BTree records and k_gapply's helpers; same contract as k_gapply: one CTA per chunk of one output
// node's triples sorted by (term, dz, dy), the sum written to the output block (or a partial slot)
// with its norms.
//
// Operator application (reference src/treebuilders/ConvolutionCalculator.cpp: applyOperator ->
// tensorXProd), grouped by line = (term, dz, dy) and plane = (term, dz):
//     out += sum_dz beta Mz(dz) [ sum_dy My(dy) [ sum_dx Mx(dx) in_(dx,dy,dz) ] ]
//
// x step (tensor cores).  One GEMM per triple, D[(y, z)][x'] += sum_x X[(y, z)][x] Mx[x'][x], with
// M = the R = (2k)^2 data rows (y, z) in tiles of 128 TMEM lanes, K = x (16 per instruction) and
// N = three column blocks of 2k: the data block is written as four and the operator as three BF16
// slices of a per-row fixed-point form (mw_slice.hpp), and the operator slices are stacked along N so that
//     data slice 0 x [m0 | m1 | m2],   data slice 1 x [0 | m0 | m1],   data slices 2, 3 x [0 | 0 | m0]
// put the products of weight 2^-16 / 2^-24 / 2^-32 (and 2^-40) into column blocks 0 / 1 / 2.  Within one
// block row blocks 0 and 1 hold exact multiples of one quantum below 2^24 quanta, so the tensor core's
// FP32 accumulation is exact there inside a triple; block 2 rounds at 2^-24 of its own size, itself
// below 2^-9 of the products.  The triples of a line accumulate in TMEM (the MMA accumulate flag), and
// the line's epilogue adds the three blocks (round to nearest) into the y step's operand.  Products
// dropped by the scheme (slice pairs of weight <= 2^-40 of the row scales), the operator's slicing
// remainder (2^-25 of its row maximum) and the data's (2^-33) are below FP32 rounding of the products;
// the data's fourth slice matters because a block's slicing error repeats in every triple that reads it.
// Staging: each triple's data image (built once per pass by k_simage) and operator image travel by one
// 1-D bulk copy each (cp.async.bulk, completion on an mbarrier) into one of two buffers; the copy for
// the next triple overlaps the current triple's MMAs.  At a line's end the MMAs of the next line's first
// triple are issued before the CUDA cores start this line's y and z steps, so both units work at once.
//
// y and z steps (CUDA cores), as in k_gapply: register-tiled GEMMs on shared operands, one thread per
// MT x NT output tile (MT = NT = 2k/4 rounded up), FP32 products; the y step sums a plane's lines in
// shared memory, the z step adds each plane (beta-scaled operator) into FP64 accumulators in TMEM.
// Operand rows use the split column layout of mw_slice.hpp, so a thread's tile row is one 16-byte load
// and one 4-byte load.
//
// Below the root the s->s block (T x T x T on the scaling part) is left out, as in k_gapply: the k^3
// correction GEMMs run on the CUDA cores (the x step's part as extra MMA columns).  Each plane's correction
// block is added into FP64 sums in TMEM by the warps that compute it, and the sums are subtracted once,
// when the chunk's block is written.
//
// Every mbarrier wait has a time limit: a wait that runs out sets the kernel's error word, and the CTA
// leaves after waiting (again with a limit) for the copies and MMAs it started.
#pragma once
#include "mw_slice.hpp"
#include "mw_umma.cuh"

namespace mwb {

// columns per correction tile: the smallest divisor d of k^2 with 2 k^2 / d tiles fitting `nthr` threads
__host__ __device__ constexpr int hc_nc(int k, int nthr) {
    int d = 1;
    while (d < k * k && ((k * k) % d != 0 || 2 * k * k / d > nthr)) ++d;
    return d;
}

template <int K>
struct HCfg {
    static constexpr int K2 = 2 * K;
    static constexpr int KP = (K2 + 3) / 4 * 4;  // 16 or 20
    static constexpr int NN = KP * KP;
    static constexpr int MT = KP / 4, NT = KP / 4;  // CUDA-core tiles of the y and z steps
    static constexpr int NTILE = NN / NT;           // column tiles: 4 KP
    static constexpr int NWARP = NTILE / 8;         // CUDA-core warps; one more warp stages and issues MMAs
    static constexpr int NTHR_S = 32 * NWARP;
    static constexpr int NTHR = NTHR_S + 32;
    static constexpr int ND = MT * NT;
    static constexpr int LDT = NN + 4;  // row stride of T1 and T2 (split column layout)
    static constexpr int MATP = KP * KP;
    // x step (image layouts in mw_slice.hpp, XGeo)
    static constexpr int R = K2 * K2;
    static constexpr int TILES = (R + 127) / 128;
    static constexpr int NCHM = K2 > 8 ? 2 : 1;  // chunks of x = 0 .. 15 per slice
    static constexpr int PACK = K2 > 16 ? 1 : 0;  // the packed step over x = 16 .. K2-1
    static constexpr int W = K2;
    static constexpr int NCOL = (3 * W + 15) / 16 * 16;
    static constexpr int IMGB = (4 * NCHM + 2 * PACK) * R * 16;  // four data slices
    static constexpr int W2 = K;  // s->s block of the x step (x', x < k; data rows y, z < k)
    static constexpr int NCOL2 = (3 * W2 + 15) / 16 * 16;
    static constexpr int NBQ = NCOL + NCOL2;  // rows of one data slice's operand: whole matrix, then s->s block
    static constexpr int OPB_Q = NCHM * NBQ * 16;
    static constexpr int OPB_A = 3 * OPB_Q;
    static constexpr int OPB_B = PACK * 2 * NCOL * 16;
    static constexpr int OPB = OPB_A + OPB_B;
    static constexpr int BUF = (IMGB + OPB + 127) / 128 * 128;
    // generated (scaling-only) inputs, and the s->s block: rows y, z < k, x < k only
    static constexpr int TILES_GEN = (K + K2 * (K - 1) + 127) / 128;
    // TMEM: lane tile t's x sums at columns tcol(t) (NCOL of them, then below the root NCOL2 s->s sums for
    // the first TILES_GEN tiles), FP64 accumulators from ACC0 (warps of one lane quarter side by side)
    static constexpr int TSTR_C = (NBQ + 31) / 32 * 32;   // tiles with s->s sums
    static constexpr int TSTR = (NCOL + 31) / 32 * 32;    // the others
    __host__ __device__ static constexpr int tcol(int t) { return t < TILES_GEN ? t * TSTR_C : TILES_GEN * TSTR_C + (t - TILES_GEN) * TSTR; }
    static constexpr int ACC0 = TILES_GEN * TSTR_C + (TILES - TILES_GEN) * TSTR;
    static constexpr int NWQ = (NWARP + 3) / 4;
    static constexpr int CS0 = ACC0 + NWQ * 2 * ND;  // FP64 sums of the s->s corrections (correction warps)
    // s->s correction of the y and z steps
    static constexpr int KK = K * K, KKK = K * K * K;
    // correction tiles (MT rows x NC columns) on the warps of lane quarters 2 and 3 only (warps 2, 3, 6, 7):
    // quarters 0 and 1 hold one more GEMM warp each when NWARP = 10
    static constexpr int NCW = 128;  // threads that take correction tiles
    static constexpr int NC = hc_nc(K, NCW);
    static constexpr int NCT = KK / NC;
    static constexpr int CSW = 2 * MT * NC;  // TMEM words of one correction thread's sums
    static constexpr int TCOLS_NEED = CS0 + 2 * CSW;  // two correction warps per lane quarter
    static constexpr int TCOLS = TCOLS_NEED <= 128 ? 128 : TCOLS_NEED <= 256 ? 256 : 512;
    static constexpr int MAXT = 372;  // triples per chunk whose 16-byte records are kept in shared memory
    static constexpr size_t SMEM = 2 * (size_t)BUF + sizeof(float) * (2 * (size_t)KP * LDT + 2 * MATP + 2 * KKK) +
                                   MAXT * 16;
    static constexpr int SMEM_STATIC = 64;  // the kernel's own __shared__ words (mbarriers, TMEM address, flag)
    // the last tile reads (TILES 128 - R) rows past the last chunk: they land in the operator image
    static constexpr bool FITS = (KP == 16 || KP == 20) && K <= 10 && K2 > 8 && NCOL <= 256 && TCOLS_NEED <= 512 &&
                                 SMEM + SMEM_STATIC <= 232448 && 2 * NCT <= NCW && 8 * KKK <= 4 * KP * LDT && NWARP >= 8 && (TILES * 128 - R) * 16 <= OPB;
};

// Block images of the tensor-core x step, one thread per data row (y, z) of a block: the row's 2k FP64
// values are contiguous in the block (x fastest), so a warp reads 32 consecutive rows as whole sectors
// straight from global memory (16-byte streaming loads, nothing staged in shared memory); the row is
// sliced (mw_slice.hpp) and written as 16-byte chunks, consecutive rows side by side.  A generated node's
// rows come from its k^3 scaling block (zero where y, z or x >= k).  Slot numbering as k_ximage.
template <int K>
__global__ void __launch_bounds__(256) k_simage(const ImgSrc* __restrict__ srcs, int nsrc, const double* __restrict__ gblk,
                                                long long nreal, long long nimg, unsigned char* __restrict__ img) {
    using C = HCfg<K>;
    constexpr int K2 = C::K2, R = C::R, NCHM = C::NCHM, BS = K2 * K2 * K2, KKK = K * K * K;
    static_assert(K2 % 2 == 0, "rows of whole 16-byte pairs");
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long slot = gid / R;
    const int r = (int)(gid - slot * R);
    if (slot >= nimg) return;
    double row[K2];
    if (slot < nreal) {
        int lo = 0, hi = nsrc - 1;  // last entry with base <= slot
        while (lo < hi) {
            const int mid = (lo + hi + 1) / 2;
            if (srcs[mid].base <= slot) lo = mid;
            else hi = mid - 1;
        }
        const ImgSrc sr = srcs[lo];
        const double2* b = reinterpret_cast<const double2*>(sr.coef + (size_t)(sr.lb + (slot - sr.base)) * BS + (size_t)r * K2);
#pragma unroll
        for (int i = 0; i < K2 / 2; ++i) {
            const double2 u = __ldcs(b + i);
            row[2 * i] = u.x;
            row[2 * i + 1] = u.y;
        }
    } else {
        const double* g = gblk + (size_t)(slot - nreal) * KKK;
        const int y = r % K2, z = r / K2;
#pragma unroll
        for (int x = 0; x < K2; ++x) row[x] = (x < K && y < K && z < K) ? g[x + K * (y + K * z)] : 0.0;
    }
    unsigned char* out = img + (size_t)slot * C::IMGB;
    auto put = [&](int chunk, const float* v) {
        uint32_t w[4];
#pragma unroll
        for (int h = 0; h < 4; ++h)
            w[h] = (uint32_t)bf16_bits_exact(v[2 * h]) | ((uint32_t)bf16_bits_exact(v[2 * h + 1]) << 16);
        *reinterpret_cast<uint4*>(out + ((size_t)chunk * R + r) * 16) = make_uint4(w[0], w[1], w[2], w[3]);
    };
    double m = 0.0;
#pragma unroll
    for (int x = 0; x < K2; ++x) m = fmax(m, fabs(row[x]));
    int e = 0;
    if (m > 0.0) frexp(m, &e);
    const double scale = ldexp(1.0, -e);
    const float inv256 = ldexpf(1.0f, e - 8);
#pragma unroll
    for (int c = 0; c < NCHM; ++c) {  // x = 8 c .. 8 c + 7 of the four slices
        float s[4][8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (8 * c + j < K2) slice4_value(row[8 * c + j], scale, inv256, s[0][j], s[1][j], s[2][j], s[3][j]);
            else s[0][j] = s[1][j] = s[2][j] = s[3][j] = 0.0f;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) put(q * NCHM + c, s[q]);
    }
    if constexpr (C::PACK) {  // [s0 | s1 | s2 | s3] of x = 16 .., four K slots per slice
        float pk[16];
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            if (16 + l < K2) slice4_value(row[16 + l], scale, inv256, pk[l], pk[4 + l], pk[8 + l], pk[12 + l]);
            else pk[l] = pk[4 + l] = pk[8 + l] = pk[12 + l] = 0.0f;
        }
        put(4 * NCHM, pk);
        put(4 * NCHM + 1, pk + 8);
    }
}

__device__ __forceinline__ float bf16_to_f32(uint16_t h) { return __uint_as_float((uint32_t)h << 16); }

// c[i][j] = sum_{k < KD} A[k][o0 + i] B[k][n0 + j] with A rows (stride LDA) in the split layout of
// MT-tiles (4 row tiles) and B rows (stride LDB) in the split layout of NT-tiles (NTILE tiles); a thread
// tile is (rt, ct).  Fully unrolled, so the loads of step k + 1 issue ahead of the FMAs of step k.  Columns
// 0-3 of the tile run as two packed FP32 pairs per row (fma.rn.f32x2, bit-identical to two fmaf), the
// fifth column as single FMAs: 15 FMA instructions per step of a 5 x 5 tile instead of 25.
// The tile's result stays packed: columns (0, 1) and (2, 3) of row i in p01[i] and p23[i], column 4 in c4[i].
template <int MT, int NT, int NTILE, int LDA, int LDB, int KD>
__device__ __forceinline__ void gemm_tile_packed(const float* __restrict__ A, const float* __restrict__ B, int rt,
                                                 int ct, unsigned long long (&p01)[MT], unsigned long long (&p23)[MT],
                                                 float (&c4)[MT]) {
    static_assert(MT == 4 || MT == 5, "tile");
    static_assert(NT == 4 || NT == 5, "tile");
#pragma unroll
    for (int i = 0; i < MT; ++i) {
        p01[i] = p23[i] = 0ull;  // (+0.0f, +0.0f)
        c4[i] = 0.0f;
    }
    const float* ap = A + 4 * rt;
    const float* a5 = A + 16 + rt;
    const float* bp = B + 4 * ct;
    const float* b5 = B + 4 * NTILE + ct;
#pragma unroll
    for (int k = 0; k < KD; ++k) {
        float a[MT];
        const float4 av = *reinterpret_cast<const float4*>(ap + k * LDA);
        a[0] = av.x;
        a[1] = av.y;
        a[2] = av.z;
        a[3] = av.w;
        if constexpr (MT == 5) a[4] = a5[k * LDA];
        const float4 bv = *reinterpret_cast<const float4*>(bp + k * LDB);
        const unsigned long long b01 = pack_f32x2(bv.x, bv.y), b23 = pack_f32x2(bv.z, bv.w);
        float b4 = 0.0f;
        if constexpr (NT == 5) b4 = b5[k * LDB];
#pragma unroll
        for (int i = 0; i < MT; ++i) {
            const unsigned long long aa = pack_f32x2(a[i], a[i]);
            p01[i] = fma_f32x2(aa, b01, p01[i]);
            p23[i] = fma_f32x2(aa, b23, p23[i]);
            if constexpr (NT == 5) c4[i] = fmaf(a[i], b4, c4[i]);
        }
    }
}
template <int MT, int NT, int NTILE, int LDA, int LDB, int KD>
__device__ __forceinline__ void gemm_tile_split(const float* __restrict__ A, const float* __restrict__ B, int rt, int ct,
                                                float (&c)[MT][NT]) {
    unsigned long long p01[MT], p23[MT];
    float c4[MT];
    gemm_tile_packed<MT, NT, NTILE, LDA, LDB, KD>(A, B, rt, ct, p01, p23, c4);
#pragma unroll
    for (int i = 0; i < MT; ++i) {
        unpack_f32x2(p01[i], c[i][0], c[i][1]);
        unpack_f32x2(p23[i], c[i][2], c[i][3]);
        if constexpr (NT == 5) c[i][4] = c4[i];
    }
}
__device__ __forceinline__ unsigned long long add_f32x2(unsigned long long a, unsigned long long b) {
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));  // two round-to-nearest adds
    return d;
}
// acc (+)= the tile's result, in packed form (bit-identical to the scalar adds)
template <int MT, int NT, int NTILE, int LDA, int LDB, int KD>
__device__ __forceinline__ void gemm_tile_split_add(const float* __restrict__ A, const float* __restrict__ B, int rt,
                                                    int ct, unsigned long long (&a01)[MT], unsigned long long (&a23)[MT],
                                                    float (&a4)[MT]) {
    unsigned long long p01[MT], p23[MT];
    float c4[MT];
    gemm_tile_packed<MT, NT, NTILE, LDA, LDB, KD>(A, B, rt, ct, p01, p23, c4);
#pragma unroll
    for (int i = 0; i < MT; ++i) {
        a01[i] = add_f32x2(a01[i], p01[i]);
        a23[i] = add_f32x2(a23[i], p23[i]);
        if constexpr (NT == 5) a4[i] += c4[i];
    }
}

// record of one triple of a chunk (16 bytes), kept in shared memory for the first MAXT triples; a
// matrix index fits 27 bits (2^27 matrices of (2k)^2 FP64 values would exceed any device memory)
struct HTri {
    int slot;  // block image slot of the input node
    int mx, my;
    unsigned mz : 27;
    unsigned flags : 5;  // HT_* below
};
static_assert(sizeof(HTri) == 16, "triple record");
enum { HT_GEN = 1, HT_LSTART = 2, HT_LEND = 4, HT_PSTART = 8, HT_PEND = 16 };

__device__ __forceinline__ void named_bar(int id, int nthr) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthr) : "memory");
}
// barrier of `nthr` threads on `id` that returns whether any of them passed a nonzero `pred`
__device__ __forceinline__ int named_bar_or(int id, int nthr, int pred) {
    int r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.s32 p, %1, 0;\n\tbar.red.or.pred q, %2, %3, p;\n\tselp.s32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"(pred), "r"(id), "r"(nthr)
        : "memory");
    return r;
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr_u32(bar)) : "memory");
}

// Warp roles: warps 0 .. NWARP-1 run the epilogues and the y and z steps (CUDA cores); warp NWARP
// (one thread) stages every triple and issues its MMAs.  mbarriers between them:
//   staged[b]   the bulk copies of buffer b landed              (producer -> producer)
//   mma_done[b] the MMAs reading buffer b completed              (tcgen05.commit -> producer)
//   line_done   the MMAs of the current line completed           (tcgen05.commit -> CUDA-core warps)
//   sums_free   the line's x sums were read out of TMEM          (one CUDA-core thread -> producer)
// Each has at most one completed phase that its waiter has not yet consumed, so parities never skip.
template <int K>
__global__ void __launch_bounds__(HCfg<K>::NTHR, 1)
    k_happly(const Chunk* __restrict__ chunks, const Item* __restrict__ items, const BTree* __restrict__ trees,
             const unsigned long long* __restrict__ tkey, const unsigned long long* __restrict__ tval,
             const int* __restrict__ csrc, const unsigned char* __restrict__ simg, long long gbase, double* partials,
             unsigned long long* ntrip_out, int* err_out) {
    using C = HCfg<K>;
    constexpr int K2 = C::K2, KP = C::KP, MT = C::MT, NT = C::NT, NTILE = C::NTILE, ND = C::ND, NC = C::NC;
    constexpr int LDT = C::LDT, MATP = C::MATP, KK = C::KK, KKK = C::KKK, R = C::R, W = C::W, W2 = C::W2;
    constexpr int NS = C::NTHR_S;
    constexpr int BS = K2 * K2 * K2;
    constexpr uint64_t kWaitNs = 2000000000ull;  // per mbarrier wait
    extern __shared__ __align__(16) unsigned char smraw[];  // 16-byte aligned: all the no-swizzle operands and bulk copies need
    __shared__ uint32_t tmem_slot;
    __shared__ __align__(8) uint64_t bars[6];  // staged[2], mma_done[2], line_done, sums_free
    __shared__ int s_bad;
    float* T1 = reinterpret_cast<float*>(smraw + 2 * (size_t)C::BUF);  // [KP][LDT], split columns
    float* T2 = T1 + KP * LDT;
    float* My = T2 + KP * LDT;  // [KP][split o]: My[b'][b] at (b, o = b')
    float* Mz = My + MATP;
    float* U1 = Mz + MATP;  // [K][K][K]
    float* U2 = U1 + KKK;
    HTri* meta = reinterpret_cast<HTri*>(U2 + KKK);
    const Chunk ch = chunks[blockIdx.x];
    const Item it = items[ch.item];
    const BTree& TR = trees[it.tree];
    const bool root = TR.root != 0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, quarter = warp & 3;
    const int ntri = ch.c1 - ch.c0;

    // the triple's input slot, operators and place in its line and plane (a line = equal key bits
    // 0..31: term << 20 | dz rank << 10 | dy rank; a plane = equal bits 10..31)
    auto load_rec = [&](int t) -> HTri {
        const unsigned long long tv = tval[t];
        const int src = csrc[(int)(tv >> 32)];
        const TermRec tr = TR.terms[(int)(tv & 0xffffffffull)];
        const uint32_t lk = (uint32_t)(tkey[t] & 0xffffffffull);
        const uint32_t lp = t > ch.c0 ? (uint32_t)(tkey[t - 1] & 0xffffffffull) : ~lk;
        const uint32_t ln = t + 1 < ch.c1 ? (uint32_t)(tkey[t + 1] & 0xffffffffull) : ~lk;
        HTri h;
        h.slot = (int)(src < 0 ? gbase + (-src - 1) : TR.img_base + (src - TR.img_lb));
        h.mx = tr.mx;
        h.my = tr.my;
        h.mz = (unsigned)tr.mz;
        h.flags = (src < 0 ? HT_GEN : 0) | (lp != lk ? HT_LSTART : 0) | (ln != lk ? HT_LEND : 0) |
                  ((lp >> 10) != (lk >> 10) ? HT_PSTART : 0) | ((ln >> 10) != (lk >> 10) ? HT_PEND : 0);
        return h;
    };
    for (int e = tid; e < min(ntri, C::MAXT); e += C::NTHR) meta[e] = load_rec(ch.c0 + e);
    auto rec = [&](int t) -> HTri { return t - ch.c0 < C::MAXT ? meta[t - ch.c0] : load_rec(t); };

    if (warp == 0) {
        tmem_alloc(&tmem_slot, C::TCOLS);
        tmem_relinquish();
    }
    if (tid == 0) {
        for (int i = 0; i < 6; ++i) mbar_init(&bars[i], 1);
        mbar_fence_init();
        s_bad = 0;
    }
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    const uint32_t tbase = tmem_slot;
    int bad = 0;

    if (warp == C::NWARP) {
        // ================= producer: staging and MMAs (one thread) =================
        if (lane == 0) {
            uint32_t fph = 0, mph = 0, dph = 0;
            bool spend[2] = {false, false}, mpend[2] = {false, false};
            const uint32_t sbase = smem_addr_u32(smraw);
            auto stage = [&](const HTri& h, int b) {
                unsigned char* dst = smraw + (size_t)b * C::BUF;
                mbar_arrive_expect_tx(&bars[b], (uint32_t)(C::IMGB + C::OPB));
                bulk_g2s(dst, simg + (size_t)h.slot * C::IMGB, C::IMGB, &bars[b]);
                bulk_g2s(dst + C::IMGB, TR.matsX + (size_t)h.mx * C::OPB, C::OPB, &bars[b]);
                spend[b] = true;
            };
            // x-step MMAs of the triple in buffer b into the line's TMEM sums, fully unrolled on descriptors
            // prepared once per buffer (start addresses in 16-byte units); a generated input is zero outside
            // its first TILES_GEN tiles and first K step, but the first triple of a line clears every tile;
            // below the root also the s->s block's sums (x', x < k; first TILES_GEN tiles)
            constexpr uint32_t idesc = umma_idesc_bf16(128, C::NCOL);
            auto issue = [&](int b, bool first, bool gen) {
                const uint32_t base = sbase + (uint32_t)(b * C::BUF);
                const uint64_t da = umma_sdesc(base, R * 16, 128);
                const uint64_t dbq = umma_sdesc(base + C::IMGB, C::NBQ * 16, 128);
                const uint64_t dq = umma_sdesc(base + C::IMGB + C::OPB_A, C::NCOL * 16, 128);
                static_for<C::TILES>([&](auto TL) {
                    constexpr int tl = decltype(TL)::value;
                    const bool live = !gen || tl < C::TILES_GEN;
                    // below the root the first tiles also take the s->s block's sums (N = NCOL + NCOL2)
                    const bool ss = !root && tl < C::TILES_GEN;
                    static_for<4>([&](auto SQ) {  // x = 0 .. 15 of data slice sq against its operand
                        constexpr int sq = decltype(SQ)::value;
                        constexpr int oq = sq < 3 ? sq : 2;  // slice 3 takes slice 2's operand
                        // operand rows (output columns) below oq W are zero for this slice: the MMA starts
                        // at the 16-row boundary below them, fewer B bytes for the same sums
                        constexpr int r0 = oq * C::W / 16 * 16;
                        static_assert(r0 <= oq * C::W && (C::NCOL - r0) % 16 == 0 && C::NCOL - r0 >= 16, "MMA N");
                        constexpr uint32_t id_full = umma_idesc_bf16(128, C::NCOL - r0);
                        constexpr uint32_t id_ss = umma_idesc_bf16(128, C::NBQ - r0);
                        const bool init = first && sq == 0;
                        if (!live && !init) return;
                        const uint64_t ad = da + (uint64_t)((sq * C::NCHM * R * 16 + tl * 2048) >> 4);
                        const uint64_t bd = dbq + (uint64_t)((oq * C::OPB_Q + r0 * 16) >> 4);
                        umma_bf16(tbase + (uint32_t)(C::tcol(tl) + r0), ad, bd, ss ? id_ss : id_full, init ? 0u : 1u);
                    });
                    if constexpr (C::PACK) {  // x = 16 .. K2-1 of all slices in one step (whole matrix only)
                        if (!gen) {
                            const uint64_t ad = da + (uint64_t)((4 * C::NCHM * R * 16 + tl * 2048) >> 4);
                            umma_bf16(tbase + (uint32_t)C::tcol(tl), ad, dq, idesc, 1u);
                        }
                    }
                });
            };
            if (ntri > 0) stage(rec(ch.c0), 0);
            if (ntri > 1) stage(rec(ch.c0 + 1), 1);
            for (int t = ch.c0; t < ch.c1; ++t) {
                const int b = (t - ch.c0) & 1;
                const HTri h = rec(t);
                const bool lstart = (h.flags & HT_LSTART) != 0;
                if (!mbar_wait(&bars[b], (fph >> b) & 1u, kWaitNs)) bad = 1;
                fph ^= 1u << b;
                spend[b] = false;
                if (!bad && lstart && t != ch.c0) {  // the previous line's sums are read out
                    if (!mbar_wait(&bars[5], dph, kWaitNs)) bad = 1;
                    dph ^= 1u;
                }
                if (bad || *reinterpret_cast<volatile int*>(&s_bad)) {
                    bad = 1;
                    break;
                }
                tmem_fence_after_sync();
                issue(b, lstart, (h.flags & HT_GEN) != 0);
                umma_commit(&bars[2 + b]);
                mpend[b] = true;
                if (h.flags & HT_LEND) umma_commit(&bars[4]);
                if (t + 2 < ch.c1) {  // refill buffer b once its MMAs are done
                    const HTri h2 = rec(t + 2);
                    if (!mbar_wait(&bars[2 + b], (mph >> b) & 1u, kWaitNs)) {
                        bad = 1;
                        break;
                    }
                    mph ^= 1u << b;
                    mpend[b] = false;
                    stage(h2, b);
                    if (t + 3 < ch.c1) prefetch_l2_bulk(simg + (size_t)rec(t + 3).slot * C::IMGB, C::IMGB);
                }
            }
            for (int b = 0; b < 2; ++b) {  // leave only after this thread's copies and MMAs have landed
                if (spend[b] && !mbar_wait(&bars[b], (fph >> b) & 1u, kWaitNs)) bad = 1;
                if (mpend[b] && !mbar_wait(&bars[2 + b], (mph >> b) & 1u, kWaitNs)) bad = 1;
            }
            if (bad) atomicExch(&s_bad, 1);
        }
        __syncwarp();
    } else {
        // ================= CUDA-core warps: epilogues, y and z steps =================
        const int rt = lane & 3, ct = warp * 8 + (lane >> 2);
        const int o0 = rt * MT, n0 = ct * NT;
        const int tb0 = n0 % KP, tc0 = n0 / KP;  // y tile: first a', c;  z tile: first a', b'
        // correction tiles: warps of lane quarters 2 and 3 (warps 2, 3, 6, 7)
        const bool cwarp = (warp & 3) >= 2 && warp < 8;
        const int cid = (((warp >> 2) << 1) | (warp & 1)) * 32 + lane;
        const int crt = cid & 1, cct = cid >> 1;
        const bool cown = !root && cwarp && cct < C::NCT;
        const int co0 = crt * MT, cn0 = cown ? cct * NC : 0;
        auto opos = [](int o) { return split_pos(o, MT, 4); };  // operator column of output index o
        const uint32_t tlane = tbase + ((uint32_t)(32 * quarter) << 16);
        const uint32_t tacc = tlane + (uint32_t)(C::ACC0 + (warp >> 2) * 2 * ND);
        // the correction warps' FP64 sums of every plane's s->s correction, subtracted once at the end
        const bool csum = !root && cwarp;  // warp-uniform (TMEM accesses are warp-collective)
        const uint32_t tcs = tlane + (uint32_t)(C::CS0 + (warp >> 2) * C::CSW);
        {
            uint32_t z[2 * ND];
#pragma unroll
            for (int q = 0; q < 2 * ND; ++q) z[q] = 0u;
            tmem_span_st<0, 2 * ND>(tacc, z);
            if (csum) tmem_span_st<0, C::CSW>(tcs, z);
        }
        auto load_mat = [&](float* dst, const float* tab, int mi) {
            constexpr int NV = MATP * 4 / 16;
            const char* src = reinterpret_cast<const char*>(tab + (size_t)mi * MATP);
            for (int e = tid; e < NV; e += NS) cp_async16(reinterpret_cast<char*>(dst) + 16 * e, src + 16 * e);
            cp_async_commit();
        };
        // whether this thread's z tile holds elements of the s->s block (c', a', b' < k; a tile never wraps
        // a row since NT divides KP)
        const bool tile_sss = o0 < K && tb0 < K && tc0 < K;
        float c2[MT][NC];
        const int nq = (C::NWARP - quarter + 3) / 4;  // warps of this lane quarter
        uint32_t lph = 0;
        bool plane_gen = true, first_line = true;
        unsigned long long ya01[MT], ya23[MT];  // the plane's y sums of this thread's tile, packed as the GEMM's
        float ya4[MT];
        bool lgen = true;
        for (int t = ch.c0; t < ch.c1; ++t) {
            const HTri h0 = rec(t);
            const bool pend = (h0.flags & HT_PEND) != 0;
            if (h0.flags & HT_PSTART) {
                plane_gen = true;
                first_line = true;
            }
            if (h0.flags & HT_LSTART) lgen = true;
            lgen = lgen && (h0.flags & HT_GEN) != 0;
            plane_gen = plane_gen && (h0.flags & HT_GEN) != 0;
            if (!(h0.flags & HT_LEND)) continue;
            named_bar(1, NS);  // readers of T1, My, U1 (last line) and of Mz, T2, U2 (last plane) are done
            load_mat(My, TR.matsS32, h0.my);
            if (pend) load_mat(Mz, TR.matsbS32, h0.mz);
            if (!mbar_wait(&bars[4], lph, kWaitNs)) bad = 1;
            bad = __any_sync(0xffffffffu, bad);  // warp-uniform: the TMEM loads below are warp-collective
            lph ^= 1u;
            tmem_fence_after_sync();
            // ---- epilogue: the line's x sums (three column blocks) -> T1 [y][x' + P z], s->s sums -> U1
            if (!bad) {
                // units of this lane quarter: the main x sums of every tile with rows here, then (below the
                // root) the s->s sums of the first tiles; round-robin over the quarter's warps
                constexpr int NU_MAX = C::TILES + C::TILES_GEN;
                const int ntl = min(C::TILES, (R - 32 * quarter + 127) / 128);  // tiles with rows in this quarter
                const int nunits = ntl + (root ? 0 : C::TILES_GEN);
#pragma unroll 1
                for (int u = warp >> 2; u < nunits && u < NU_MAX; u += nq) {
                    if (u < ntl) {
                        const int tl = u;
                        uint32_t v[3 * W];
                        tmem_span_ld<0, 3 * W>(tlane + (uint32_t)C::tcol(tl), v);
                        tmem_span_wait<0, 3 * W>(v);
                        const int r = 128 * tl + 32 * quarter + lane;
                        if (r < R) {
                            const int y = r % K2, z = r / K2;
                            float o[KP];
#pragma unroll
                            for (int x = 0; x < KP; ++x)
                                o[x] = x < W ? __uint_as_float(v[x]) + (__uint_as_float(v[W + x]) + __uint_as_float(v[2 * W + x]))
                                             : 0.0f;
                            float* row = T1 + y * LDT;
                            constexpr int TPR = KP / NT;  // column tiles per z
#pragma unroll
                            for (int uu = 0; uu < TPR; ++uu)
                                *reinterpret_cast<float4*>(row + 4 * (TPR * z + uu)) =
                                    make_float4(o[NT * uu], o[NT * uu + 1], o[NT * uu + 2], o[NT * uu + 3]);
                            if constexpr (NT == 5)
                                *reinterpret_cast<float4*>(row + 4 * NTILE + TPR * z) = make_float4(o[4], o[9], o[14], o[19]);
                        }
                    } else {
                        const int tl = u - ntl;
                        uint32_t v[3 * W2];
                        tmem_span_ld<0, 3 * W2>(tlane + (uint32_t)(C::tcol(tl) + C::NCOL), v);
                        tmem_span_wait<0, 3 * W2>(v);
                        const int r = 128 * tl + 32 * quarter + lane;
                        const int y = r % K2, z = r / K2;
                        if (y < K && z < K) {
#pragma unroll
                            for (int x = 0; x < W2; ++x)
                                U1[y * KK + x + K * z] =
                                    __uint_as_float(v[x]) + (__uint_as_float(v[W2 + x]) + __uint_as_float(v[2 * W2 + x]));
                        }
                    }
                }
            }
            tmem_fence_before_sync();
            cp_async_wait_all();
            bad = named_bar_or(1, NS, bad || *reinterpret_cast<volatile int*>(&s_bad));  // T1, U1, My, Mz are in
            if (tid == 0) mbar_arrive(&bars[5]);  // the producer may start the next line's MMAs
            if (bad) break;
            // ---- y: T2[c][a' + P b'] (+)= sum_b My[b'][b] T1[b][a' + P c]   (a plane sums its lines)
            {
                // this thread's y tile, summed over the plane's lines in registers (a tile of a generated
                // line is zero when its z index c >= k)
                if (first_line) {
#pragma unroll
                    for (int i = 0; i < MT; ++i) {
                        ya01[i] = ya23[i] = 0ull;
                        ya4[i] = 0.0f;
                    }
                }
                if (!(lgen && !(tc0 < K))) {
                    if (lgen) gemm_tile_split_add<MT, NT, NTILE, KP, LDT, K>(My, T1, rt, ct, ya01, ya23, ya4);
                    else gemm_tile_split_add<MT, NT, NTILE, KP, LDT, K2>(My, T1, rt, ct, ya01, ya23, ya4);
                }
                if (pend) {  // the plane's y sums -> T2[c][a' + P b'] for the z step
                    float* row = T2 + tc0 * LDT;
#pragma unroll
                    for (int i = 0; i < MT; ++i) {
                        const int m = tb0 + KP * (o0 + i);  // column a' + P b' of the tile's first value
                        float y0, y1, y2, y3;
                        unpack_f32x2(ya01[i], y0, y1);
                        unpack_f32x2(ya23[i], y2, y3);
                        *reinterpret_cast<float4*>(row + 4 * (m / NT)) = make_float4(y0, y1, y2, y3);
                        if constexpr (NT == 5) row[4 * NTILE + m / NT] = ya4[i];
                    }
                }
            }
            if (cown) {  // U2[c][a' + k b'] (+)= sum_{b<k} Ty[b'][b] U1[b][a' + k c]
                float cc[MT][NC];
#pragma unroll
                for (int i = 0; i < MT; ++i)
#pragma unroll
                    for (int j = 0; j < NC; ++j) cc[i][j] = 0.0f;
                for (int b = 0; b < K; ++b) {
#pragma unroll
                    for (int i = 0; i < MT; ++i) {
                        const float m = My[b * KP + opos(co0 + i)];
#pragma unroll
                        for (int j = 0; j < NC; ++j) cc[i][j] = fmaf(m, U1[b * KK + cn0 + j], cc[i][j]);
                    }
                }
#pragma unroll
                for (int i = 0; i < MT; ++i)
#pragma unroll
                    for (int j = 0; j < NC; ++j) {
                        const int n = cn0 + j;
                        if (co0 + i < K) {
                            float& d = U2[(n / K) * KK + (n % K) + K * (co0 + i)];
                            d = first_line ? cc[i][j] : d + cc[i][j];
                        }
                    }
            }
            first_line = false;
            if (!pend) continue;
            named_bar(1, NS);  // T2 and U2 of the plane are complete
            // ---- z: acc[c'][a' + P b'] += sum_c (beta Mz)[c'][c] T2[c][a' + P b']  (- previous correction)
            {
                // FP64 accumulators in TMEM: one read of all this thread's words, issued ahead of the GEMM
                // (the previous plane's write back completes first), one write back
                uint32_t r[2 * ND];
                tmem_wait_st();
                tmem_span_ld<0, 2 * ND>(tacc, r);
                float c[MT][NT];
                if (plane_gen) gemm_tile_split<MT, NT, NTILE, KP, LDT, K>(Mz, T2, rt, ct, c);
                else gemm_tile_split<MT, NT, NTILE, KP, LDT, K2>(Mz, T2, rt, ct, c);
                tmem_span_wait<0, 2 * ND>(r);
#pragma unroll
                for (int i = 0; i < MT; ++i)
#pragma unroll
                    for (int j = 0; j < NT; ++j) {
                        const int d = i * NT + j;
                        double_to_words(words_to_double(r[2 * d], r[2 * d + 1]) + (double)c[i][j], r[2 * d], r[2 * d + 1]);
                    }
                tmem_span_st<0, 2 * ND>(tacc, r);
            }
            if (cown) {  // c2[c'][a' + k b'] = sum_{c<k} (beta Tz)[c'][c] U2[c][a' + k b']
#pragma unroll
                for (int i = 0; i < MT; ++i)
#pragma unroll
                    for (int j = 0; j < NC; ++j) c2[i][j] = 0.0f;
                for (int cz = 0; cz < K; ++cz) {
#pragma unroll
                    for (int i = 0; i < MT; ++i) {
                        const float m = Mz[cz * KP + opos(co0 + i)];
#pragma unroll
                        for (int j = 0; j < NC; ++j) c2[i][j] = fmaf(m, U2[cz * KK + cn0 + j], c2[i][j]);
                    }
                }
            }
            if (csum) {  // add the plane's correction block into this thread's FP64 sums
                uint32_t w[C::CSW];
                tmem_wait_st();
                tmem_span_ld<0, C::CSW>(tcs, w);
                tmem_span_wait<0, C::CSW>(w);
                if (cown) {
#pragma unroll
                    for (int i = 0; i < MT; ++i)
#pragma unroll
                        for (int j = 0; j < NC; ++j) {
                            const int q = 2 * (i * NC + j);
                            double_to_words(words_to_double(w[q], w[q + 1]) + (double)c2[i][j], w[q], w[q + 1]);
                        }
                }
                tmem_span_st<0, C::CSW>(tcs, w);
            }
        }
        cp_async_wait_all();
        named_bar(1, NS);  // T1 is no longer read: it takes the s->s correction sums (FP64 [c'][a' + k b'])
        double* Usum = reinterpret_cast<double*>(T1);
        if (!bad && csum) {
            uint32_t w[C::CSW];
            tmem_wait_st();
            tmem_span_ld<0, C::CSW>(tcs, w);
            tmem_span_wait<0, C::CSW>(w);
            if (cown) {
#pragma unroll
                for (int i = 0; i < MT; ++i)
#pragma unroll
                    for (int j = 0; j < NC; ++j)
                        if (co0 + i < K) Usum[(co0 + i) * KK + cn0 + j] = words_to_double(w[2 * (i * NC + j)], w[2 * (i * NC + j) + 1]);
            }
        }
        named_bar(1, NS);
        if (!bad) {
            double* dst = ch.slot < 0 ? TR.ocoef + (size_t)it.node * BS : partials + (size_t)ch.slot * BS;
            double n2 = 0.0, w2 = 0.0;
            uint32_t r[2 * ND];
            tmem_wait_st();
            tmem_span_ld<0, 2 * ND>(tacc, r);
            tmem_span_wait<0, 2 * ND>(r);
#pragma unroll
            for (int i = 0; i < MT; ++i)
#pragma unroll
                for (int j = 0; j < NT; ++j) {
                    const int d = i * NT + j;
                    double v = words_to_double(r[2 * d], r[2 * d + 1]);
                    const int cz = o0 + i, ax = tb0 + j, by = tc0;
                    if (!root && tile_sss && cz < K && ax < K) v -= Usum[cz * KK + ax + K * by];
                    if (cz < K2 && ax < K2 && by < K2) {
                        dst[ax + K2 * (by + K2 * cz)] = v;
                        n2 += v * v;
                        if (!(ax < K && by < K && cz < K)) w2 += v * v;
                    }
                }
            // per-warp partial norms into T2 (no longer read)
            for (int o = 16; o; o >>= 1) {
                n2 += __shfl_down_sync(0xffffffffu, n2, o);
                w2 += __shfl_down_sync(0xffffffffu, w2, o);
            }
            if (lane == 0) {
                reinterpret_cast<double*>(T2)[warp] = n2;
                reinterpret_cast<double*>(T2)[32 + warp] = w2;
            }
        }
    }
    tmem_fence_before_sync();
    bad = __syncthreads_or(bad || s_bad);
    tmem_fence_after_sync();
    if (warp == 0) tmem_dealloc(tbase, C::TCOLS);
    if (bad) {
        if (tid == 0) atomicExch(err_out, 1);
        return;
    }
    if (tid == 0) {
        double n2 = 0.0, w2 = 0.0;
        for (int w = 0; w < C::NWARP; ++w) {
            n2 += reinterpret_cast<const double*>(T2)[w];
            w2 += reinterpret_cast<const double*>(T2)[32 + w];
        }
        if (ch.slot < 0) {
            TR.onorm2[it.node] = n2;
            TR.ownorm2[it.node] = w2;
        }
        atomicAdd(ntrip_out, (unsigned long long)ntri);
    }
}
}  // namespace mwb
