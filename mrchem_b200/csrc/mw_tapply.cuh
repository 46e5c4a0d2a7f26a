// mw_tapply.cuh -- the contraction of the NS-form apply on the fifth-generation tensor cores
// (tcgen05.mma kind::tf32, split-TF32 products, FP32 sums inside a term, compensated summation over
// terms).  Included by mw_apply.cu after the Chunk / Item / BTree records; same contract as k_gapply:
// one CTA per chunk of (input node, term) pairs of one output node, the sum written to the output
// block (or a partial slot) together with its norms.
//
// Operator application of one term (reference src/treebuilders/ConvolutionCalculator.cpp:
// applyOperator -> tensorXProd), with the 2k x 2k NS matrices Mx, My, Mz (Mz scaled by the term's beta):
//      out[a'][b'][c'] = sum_{a,b,c} Mx[a'][a] My[b'][b] Mz[c'][c] in[a][b][c]
// done as three GEMMs D = A B^T with M = the two free indices (rows, one TMEM lane each), N = the
// output index, K = the contracted index:
//      step x: rows (b, c),  slot  b + S1 c      D1[slot][a'] = sum_a X[slot][a] Mx[a'][a]
//      step y: rows (c, a'), slot  c + S2 a'     D2[slot][b'] = sum_b T1[slot][b] My[b'][b]
//      step z: rows (a', b'), slot a' + S3 b'    D3[slot][c'] = sum_c T2[slot][c] Mz[c'][c]
// Every operand is K-major in shared memory (element (slot, k) at 16 (slot + MR (k / 4)) + 4 (k % 4),
// with a chunk stride MR per operand).
// The epilogue of a step reads its row of D from TMEM (thread = TMEM lane = slot), transposes 4 x 4
// blocks inside each quad of lanes (four consecutive slots share the slow index and hold four
// consecutive values of the next step's contracted index), splits the values into TF32 hi + lo and
// stores 16 bytes per lane into the next step's operand.  The operators are split into three TF32
// pieces (hi + mid + lo, about 33 bits) and the products are taken in two MMAs per K step with
// N = 3 KP8 (an MMA costs about the same for any N up to 64 columns):
//      D  = A_hi [B_hi; B_mid; B_lo]^T      D += A_lo [0; B_hi; B_mid]^T
// so that columns 0 .. KP8 hold the hi*hi sum alone (the second MMA adds exact zeros there) and the
// small products (hi*mid, hi*lo, lo*hi, lo*mid) collect in the other two thirds.  The tensor core's
// FP32 accumulation truncates; the large sum takes one accumulation per K step and the thirds are added
// with round-to-nearest in the epilogue.  The operators of a term sit in one shared K-major image of
// 12 KP8 rows [0; Mx_hi; Mx_mid; Mx_lo; 0; My_...; 0; Mz_...] read through 3 KP8-row windows; each
// step's rows are reloaded (cp.async) for the next term as soon as that step's MMAs have completed.
// The z result of each term goes into the node's accumulator in TMEM: an FP32 pair (hi, lo) per value
// updated by an error-free two-sum (compensated summation over terms), converted to FP64 once at the
// end.  Two warps share each TMEM lane quarter and split the columns of every epilogue.
//
// Below the root the s->s block must be left out (the NS form has no T term there): the scaling part
// of out gets  sum_t (Mx_ss x My_ss x Mz_ss) in_sss  subtracted.  Those k x k x k GEMMs run on the
// CUDA cores of the same CTA while the tensor core works on the full step (threads < k^2, FP32
// products, FP64 sums over terms, subtracted once at the end).
//
// Synchronisation per term: two mbarriers per step (the first half of the tiles, the rest), armed by
// tcgen05.commit from the issuing thread and waited for by all threads with a time limit (a wait that
// runs out sets the kernel's error word and every thread leaves through the same barriers), so that
// the epilogue of the first tiles runs while the tensor core works on the others (x and z steps; the
// y epilogue writes over the y MMAs' own operand and waits for both); every mbarrier
// completes once per term, so one phase bit serves all six.  A CTA barrier after each epilogue
// publishes the new operand (fence.proxy.async) and orders the TMEM reads before the next MMAs
// (tcgen05.fence::before_thread_sync / after_thread_sync).
#pragma once
#include "mw_umma.cuh"

namespace mwb {

template <int K>
struct TCfg {
    static constexpr int NTHR = 256;
    static constexpr int K2 = 2 * K;
    static constexpr int KP4 = (K2 + 3) / 4 * 4;  // contracted index padded to whole 16-byte chunks
    static constexpr int KP8 = (K2 + 7) / 8 * 8;  // padded to whole K steps
    static constexpr int NCH = KP8 / 4;
    static constexpr int NKS = KP8 / 8;       // K steps, full blocks
    static constexpr int NKSG = (K + 7) / 8;  // K steps, generated (scaling-only) blocks
    static constexpr int NG = (K2 + 3) / 4;   // 4-column groups of an epilogue row
    static constexpr int NGH = (NG + 1) / 2;  // groups per warp half
    static constexpr int S1 = KP4, S2 = KP4, S3 = K2 + 1;
    static constexpr int R1 = S1 * (K2 - 1) + KP4;  // slots each step's MMAs must cover
    static constexpr int R2 = S2 * (K2 - 1) + KP4;
    static constexpr int R3 = S3 * (K2 - 1) + K2;
    static constexpr int T1 = (R1 + 127) / 128, T2 = (R2 + 127) / 128, T3 = (R3 + 127) / 128;
    static constexpr int RMAX = R1 > R2 ? (R1 > R3 ? R1 : R3) : (R2 > R3 ? R2 : R3);
    static constexpr int NTM = (RMAX + 127) / 128;
    // row strides of the K chunks (>= every slot written), chosen for the epilogue that writes the
    // operand: the y epilogue (z operand) is conflict-free with a stride of 4 mod 8; the x epilogue (y
    // operand) puts a quad's lanes j and j+2 in one bank group whatever the stride, and a stride of
    // 2 mod 8 keeps the two quads of an 8-lane phase in different groups.  The input operand uses MR.
    static constexpr int MR = (RMAX + 3) / 8 * 8 + 4;
    static constexpr int MRY = (R2 + 5) / 8 * 8 + 2;
    static constexpr int MRMAX = MR > MRY ? MR : MRY;
    static constexpr int IMG = 16 * (MRMAX * (NCH - 1) + 128 * NTM);  // bytes of one operand image
    static constexpr int NB = 12 * KP8;                             // rows of the shared operator image
    static constexpr int OPIMG = NB * KP8 * 4;                      // its bytes
    static constexpr int GOPB = 3 * KP8 * KP8 * 4;  // one global operator image (hi, mid, lo rows)
    static constexpr int NMMA = 3 * KP8;            // MMA N
    static constexpr int ATF = KP4 * KP4;           // FP32 transposed table (floats)
    static constexpr int KK = K * K, KKK = K * K * K;
    static constexpr int ACCW = 2 * K2;                 // accumulator words (FP32 hi, lo) per slot and tile
    static constexpr int DSTR = (NMMA + 15) / 16 * 16;  // TMEM columns per tile of D
    static constexpr int COL_D = 0, COL_ACC = NTM * DSTR;
    static constexpr int TCOLS_NEED = COL_ACC + NTM * ACCW;
    static constexpr int TCOLS = TCOLS_NEED <= 128 ? 128 : TCOLS_NEED <= 256 ? 256 : 512;
    static constexpr size_t SMEM = 4 * (size_t)IMG + (size_t)OPIMG + 3 * (size_t)ATF * 4 + 3 * (size_t)KKK * 4;
    static constexpr bool FITS = SMEM + 1024 <= 232448 && TCOLS_NEED <= 512 && KK <= 128 && KP8 >= 16 &&
                                 NMMA <= 256 && (size_t)IMG >= (size_t)KKK * 8 + 64 * 8 && MRMAX < 16384;
};

template <int K>
__global__ void __launch_bounds__(256, 1)
    k_tapply(const Chunk* __restrict__ chunks, const Item* __restrict__ items, const BTree* __restrict__ trees,
             const int* __restrict__ cdelta, const int* __restrict__ csrc, const double* __restrict__ gblk,
             const double* __restrict__ gnorm2, double* partials, unsigned long long* ntrip_out, int* err_out) {
    using C = TCfg<K>;
    constexpr int NTHR = C::NTHR;
    constexpr int K2 = C::K2, KP4 = C::KP4, KP8 = C::KP8, MR = C::MR, MRY = C::MRY, KK = C::KK, KKK = C::KKK;
    constexpr int S1 = C::S1, S2 = C::S2, S3 = C::S3, ACCW = C::ACCW, IMG = C::IMG;
    constexpr int NB = C::NB, GOPB = C::GOPB, ATF = C::ATF, NG = C::NG, NGH = C::NGH, DSTR = C::DSTR;
    constexpr int BS = K2 * K2 * K2;
    constexpr uint64_t kWaitNs = 2000000000ull;  // per mbarrier wait
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ __align__(8) uint64_t bars[6];
    __shared__ uint32_t tmem_slot;
    unsigned char* xh = smraw;  // step-x operand, hi and lo images (the input block), then T hi, T lo
    unsigned char* ops = smraw + 4 * IMG;                   // operator image, NB rows
    float* ats = reinterpret_cast<float*>(ops + C::OPIMG);  // [3][ATF] FP32 At[k][o] (s->s correction)
    float* xs = ats + 3 * ATF;                              // xs[a KK + b + K c] = in_sss
    float* u1 = xs + KKK;                                   // u1[b KK + c + K a']
    float* u2 = u1 + KKK;                                   // u2[c KK + a' + K b']
    const uint32_t sxh = smem_addr_u32(xh), sxl = sxh + IMG, sth = sxh + 2 * IMG, stl = sxh + 3 * IMG;
    const uint32_t sops = smem_addr_u32(ops);

    const Chunk ch = chunks[blockIdx.x];
    const Item it = items[ch.item];
    const BTree& TR = trees[it.tree];
    const float* at32 = TR.matsT32;
    const float* atb32 = TR.matsbT32;
    const bool root = TR.root != 0;
    const double theta = TR.theta;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, j4 = lane & 3;
    const int quarter = warp & 3, half = warp >> 2;  // TMEM lane quarter; which columns of it

    // operand and operator images start zero: padding chunks, the operator image's zero rows and slots
    // that no step writes stay finite
    for (int e = tid; e < (4 * IMG + C::OPIMG) / 16; e += NTHR) st_shared_v4(sxh + 16 * e, 0u, 0u, 0u, 0u);
    if (tid == 0) {
        for (int q = 0; q < 6; ++q) mbar_init(&bars[q], 1);
        mbar_fence_init();
    }
    if (warp == 0) {
        tmem_alloc(&tmem_slot, C::TCOLS);
        tmem_relinquish();
    }
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    const uint32_t tbase = tmem_slot;
    const uint32_t tlane = tbase + ((uint32_t)(32 * quarter) << 16);
    {
        uint32_t z[2 * K];
#pragma unroll
        for (int q = 0; q < 2 * K; ++q) z[q] = 0u;
        for (int t = 0; t < C::NTM; ++t) tmem_span_st<0, 2 * K>(tlane + C::COL_ACC + ACCW * t + 2 * K * half, z);
        tmem_wait_st();
    }
    double corr[K];
#pragma unroll
    for (int q = 0; q < K; ++q) corr[q] = 0.0;
    unsigned long long ntrip = 0;
    uint32_t ph = 0;  // parity of the current term's phase of every mbarrier
    int bad = 0;
    constexpr uint32_t idesc = umma_idesc_tf32(128, C::NMMA);

    // operator of step q (0 x, 1 y, 2 z) of a term into its rows of the image (and, below the root, its
    // FP32 s->s table); the copies complete at the next cp_async_wait_all
    auto load_op = [&](int q, const TermRec& tr) {
        const int mi = q == 0 ? tr.mx : q == 1 ? tr.my : tr.mz;
        const unsigned char* src = reinterpret_cast<const unsigned char*>(q == 2 ? TR.matsbI : TR.matsI) +
                                   (size_t)mi * GOPB;
        const int r0 = KP8 + 4 * KP8 * q;
        for (int e = tid; e < 3 * KP8 * (KP8 / 4); e += NTHR) {
            const int n = e % (3 * KP8), j = e / (3 * KP8);
            cp_async16(ops + 16 * (r0 + n + NB * j), src + 16 * e);
        }
        if (!root) {
            const float* at = (q == 2 ? atb32 : at32) + (size_t)mi * ATF;
            for (int e = tid; e < ATF / 4; e += NTHR) cp_async16(ats + q * ATF + 4 * e, at + 4 * e);
        }
        cp_async_commit();
    };
    // one step: every tile of 128 slots, every K step, two MMAs (A_hi against [hi; mid; lo], A_lo against
    // [0; hi; mid] of the operator); consecutive MMAs go to different tiles (independent accumulators);
    // the first half of the tiles commits to bar2[0], the rest to bar2[1]
    auto issue = [&](uint32_t a_hi, uint32_t a_lo, int mra, int q, int ntiles, int nks, uint64_t* bar2) {
        tmem_fence_after_sync();
        const uint32_t r0 = (uint32_t)(KP8 + 4 * KP8 * q);
        const uint64_t ah0 = umma_sdesc(a_hi, 16u * mra, 128u), al0 = umma_sdesc(a_lo, 16u * mra, 128u);
        const uint64_t b1 = umma_sdesc(sops + 16u * r0, 16u * NB, 128u);
        const uint64_t b2 = umma_sdesc(sops + 16u * (r0 - KP8), 16u * NB, 128u);
        const int nfirst = (ntiles + 1) / 2;
        for (int part = 0; part < 2; ++part) {
            const int t0 = part == 0 ? 0 : nfirst, t1 = part == 0 ? nfirst : ntiles;
            for (int kk = 0; kk < nks; ++kk) {
                const uint32_t acc = kk > 0 ? 1u : 0u;
                const uint64_t bo = (uint64_t)(NB * 2 * kk);  // descriptor start addresses are in 16-byte units
                for (int t = t0; t < t1; ++t)
                    umma_tf32(tbase + (uint32_t)(C::COL_D + DSTR * t), ah0 + (uint64_t)(128 * t + mra * 2 * kk),
                              b1 + bo, idesc, acc);
                for (int t = t0; t < t1; ++t)
                    umma_tf32(tbase + (uint32_t)(C::COL_D + DSTR * t), al0 + (uint64_t)(128 * t + mra * 2 * kk),
                              b2 + bo, idesc, 1u);
            }
            umma_commit(&bar2[part]);  // arrives when this part's MMAs (and all earlier ones) are done
        }
    };
    // epilogue of the x or y step: slot (fast, slow) with fast = slot % S, slow = slot / S holds the
    // values of output index `col`; the next operand takes slot next_slot(slow, col), K chunk fast / 4.
    // This warp takes the column groups g = half, half + 2, ...
    auto epi = [&](auto s_tag, int mrn, int t0, int t1, auto next_slot) {
        constexpr int S = decltype(s_tag)::value;
        for (int t = t0; t < t1; ++t) {
            uint32_t r[12 * NGH];
            static_for<NGH>([&](auto gi_c) {
                constexpr int gi = decltype(gi_c)::value;
                const int g = half + 2 * gi;
                if (g < NG) {
                    const uint32_t a = tlane + (uint32_t)(C::COL_D + DSTR * t + 4 * g);
                    tmem_span_ld<12 * gi, 4>(a, r);
                    tmem_span_ld<12 * gi + 4, 4>(a + KP8, r);
                    tmem_span_ld<12 * gi + 8, 4>(a + 2 * KP8, r);
                }
            });
            tmem_span_wait<0, 12 * NGH>(r);
            const int m = 128 * t + 32 * quarter + lane;
            const int fast = m % S, slow = m / S;
            const bool rowok = fast < K2 && slow < K2;
            const int chunk = (fast - j4) >> 2;
#pragma unroll
            for (int gi = 0; gi < NGH; ++gi) {
                const int g = half + 2 * gi;
                if (g >= NG) break;
                float x[4];
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    x[q] = rowok ? __uint_as_float(r[12 * gi + q]) +
                                       (__uint_as_float(r[12 * gi + 4 + q]) + __uint_as_float(r[12 * gi + 8 + q]))
                                 : 0.0f;
                quad_transpose(x, j4);
                const int col = 4 * g + j4;
                if (slow < K2 && col < K2) {
                    const uint32_t off = 16u * (uint32_t)(next_slot(slow, col) + mrn * chunk);
                    uint32_t h[4], l[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) split_tf32(x[q], h[q], l[q]);
                    st_shared_v4(sth + off, h[0], h[1], h[2], h[3]);
                    st_shared_v4(stl + off, l[0], l[1], l[2], l[3]);
                }
            }
        }
    };
    // epilogue of the z step: accumulator pair (hi, lo) += D3 row by two-sum, columns c' of this half
    auto epi_z = [&](int t0, int t1) {
        for (int t = t0; t < t1; ++t) {
            uint32_t d[3 * K], a[2 * K];
            const uint32_t td = tlane + (uint32_t)(C::COL_D + DSTR * t + K * half);
            tmem_span_ld<0, K>(td, d);
            tmem_span_ld<K, K>(td + KP8, d);
            tmem_span_ld<2 * K, K>(td + 2 * KP8, d);
            const uint32_t ta = tlane + (uint32_t)(C::COL_ACC + ACCW * t + 2 * K * half);
            tmem_span_ld<0, 2 * K>(ta, a);
            tmem_span_wait<0, 3 * K>(d);
            tmem_span_wait<0, 2 * K>(a);
            const int m = 128 * t + 32 * quarter + lane;
            if ((m % S3) < K2 && (m / S3) < K2) {
#pragma unroll
                for (int c = 0; c < K; ++c) {
                    const float v = __uint_as_float(d[c]) + (__uint_as_float(d[K + c]) + __uint_as_float(d[2 * K + c]));
                    const float ah = __uint_as_float(a[2 * c]);
                    const float sum = ah + v;
                    const float bv = sum - ah;
                    const float err = (ah - (sum - bv)) + (v - bv);
                    a[2 * c] = __float_as_uint(sum);
                    a[2 * c + 1] = __float_as_uint(__uint_as_float(a[2 * c + 1]) + err);
                }
            }
            tmem_span_st<0, 2 * K>(ta, a);
        }
        tmem_wait_st();
    };
    // s->s correction on the CUDA cores (threads < k^2)
    auto corr_x = [&]() {  // u1[b KK + c + K a'] = sum_{a<k} Mx[a'][a] xs[a KK + b + K c]
        if (root || tid >= KK) return;
        const float* A = ats;
        float s[K];
#pragma unroll
        for (int o = 0; o < K; ++o) s[o] = 0.0f;
        for (int a = 0; a < K; ++a) {
            const float xv = xs[a * KK + tid];
#pragma unroll
            for (int o = 0; o < K; ++o) s[o] = fmaf(A[a * KP4 + o], xv, s[o]);
        }
        const int b = tid % K, c = tid / K;
#pragma unroll
        for (int o = 0; o < K; ++o) u1[b * KK + c + K * o] = s[o];
    };
    auto corr_y = [&]() {  // u2[c KK + a' + K b'] = sum_{b<k} My[b'][b] u1[b KK + c + K a']
        if (root || tid >= KK) return;
        const float* A = ats + ATF;
        float s[K];
#pragma unroll
        for (int o = 0; o < K; ++o) s[o] = 0.0f;
        for (int b = 0; b < K; ++b) {
            const float v = u1[b * KK + tid];
#pragma unroll
            for (int o = 0; o < K; ++o) s[o] = fmaf(A[b * KP4 + o], v, s[o]);
        }
        const int c = tid % K, ap = tid / K;
#pragma unroll
        for (int o = 0; o < K; ++o) u2[c * KK + ap + K * o] = s[o];
    };
    auto corr_z = [&]() {  // corr[c'] += sum_{c<k} (beta Mz)[c'][c] u2[c KK + a' + K b']
        if (root || tid >= KK) return;
        const float* A = ats + 2 * ATF;
        float s[K];
#pragma unroll
        for (int o = 0; o < K; ++o) s[o] = 0.0f;
        for (int c = 0; c < K; ++c) {
            const float v = u2[c * KK + tid];
#pragma unroll
            for (int o = 0; o < K; ++o) s[o] = fmaf(A[c * KP4 + o], v, s[o]);
        }
#pragma unroll
        for (int o = 0; o < K; ++o) corr[o] += (double)s[o];
    };
    // the input block: slot b + S1 c, K chunk a / 4 (FP64 -> FP32 -> TF32 hi + lo); in_sss into xs
    // (every thread first issues the loads of UNR items, then converts and stores them)
    auto load_x = [&](const double* blk, bool gen) {
        constexpr int NQ = KP4 / 4, NROW = S1 * K2, NIT = (NROW * NQ + NTHR - 1) / NTHR, UNR = 4;
        for (int i0 = 0; i0 < NIT; i0 += UNR) {
            double d[UNR][4];
#pragma unroll
            for (int u = 0; u < UNR; ++u) {
                const int e = tid + NTHR * (i0 + u);
                const int row = e % NROW, q = e / NROW;
                const int b = row % S1, c = row / S1;
#pragma unroll
                for (int i = 0; i < 4; ++i) d[u][i] = 0.0;
                if (e < NROW * NQ && b < K2) {
                    if (gen) {
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const int a = 4 * q + i;
                            if (a < K && b < K && c < K) d[u][i] = blk[a + K * (b + K * c)];
                        }
                    } else {
                        // K2 is even: the pairs (a, a+1), a even, are 16-byte aligned
                        const double2* p2 = reinterpret_cast<const double2*>(blk + 4 * q + K2 * (b + K2 * c));
                        const double2 v0 = p2[0];
                        d[u][0] = v0.x;
                        d[u][1] = v0.y;
                        if (4 * q + 2 < K2) {
                            const double2 v1 = p2[1];
                            d[u][2] = v1.x;
                            d[u][3] = v1.y;
                        }
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < UNR; ++u) {
                const int e = tid + NTHR * (i0 + u);
                if (e >= NROW * NQ) continue;
                const int row = e % NROW, q = e / NROW;
                const int b = row % S1, c = row / S1;
                float v[4];
                uint32_t h[4], l[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int a = 4 * q + i;
                    v[i] = (float)d[u][i];
                    if (!root && a < K && b < K && c < K) xs[a * KK + b + K * c] = v[i];
                    split_tf32(v[i], h[i], l[i]);
                }
                const uint32_t off = 16u * (uint32_t)(row + MR * q);
                st_shared_v4(sxh + off, h[0], h[1], h[2], h[3]);
                st_shared_v4(sxl + off, l[0], l[1], l[2], l[3]);
            }
        }
    };

    for (int ci = ch.c0; ci < ch.c1 && !bad; ++ci) {
        const int src = csrc[ci];
        const bool gen = src < 0;
        const double nu = gen ? sqrt(gnorm2[-src - 1]) : sqrt(TR.in.norm2[src]);
        const DeltaRec de = TR.deltas[cdelta[ci]];
        if (!(nu > 0.0) || de.maxb * nu < theta) continue;
        if (TR.terms[de.t0].bound * nu < theta) continue;
        if (tid == 0 && ci + 1 < ch.c1) {  // the next candidate's block: into L2 while this one runs
            const int s1 = csrc[ci + 1];
            if (s1 < 0) prefetch_l2_bulk(gblk + (size_t)(-s1 - 1) * KKK, (unsigned)(KKK * sizeof(double)));
            else prefetch_l2_bulk(TR.in.coef + (size_t)s1 * BS, (unsigned)(BS * sizeof(double)));
        }
        // every reader of the previous block and operators is done (barrier at the end of each term)
        load_x(gen ? gblk + (size_t)(-src - 1) * KKK : TR.in.coef + (size_t)src * BS, gen);
        {
            const TermRec t0 = TR.terms[de.t0];
            load_op(0, t0);
            load_op(1, t0);
            load_op(2, t0);
        }
        cp_async_wait_all();
        fence_proxy_async_smem();
        bad = __syncthreads_or(bad);
        if (bad) break;
        const int nks = gen ? C::NKSG : C::NKS;
        for (int ti = de.t0; ti < de.t1; ++ti) {
            const TermRec tr = TR.terms[ti];
            if (tr.bound * nu < theta) break;
            const bool has_next = ti + 1 < de.t1 && !(TR.terms[ti + 1].bound * nu < theta);
            const TermRec tn = has_next ? TR.terms[ti + 1] : tr;
            // ---- x
            if (tid == 0) issue(sxh, sxl, MR, 0, C::T1, nks, &bars[0]);
            corr_x();
            if (!mbar_wait(&bars[0], ph, kWaitNs)) bad = 1;
            tmem_fence_after_sync();
            epi(std::integral_constant<int, S1>{}, MRY, 0, (C::T1 + 1) / 2, [](int c, int ap) { return c + S2 * ap; });
            if (!mbar_wait(&bars[1], ph, kWaitNs)) bad = 1;
            tmem_fence_after_sync();
            epi(std::integral_constant<int, S1>{}, MRY, (C::T1 + 1) / 2, C::T1, [](int c, int ap) { return c + S2 * ap; });
            tmem_fence_before_sync();
            cp_async_wait_all();
            fence_proxy_async_smem();
            bad = __syncthreads_or(bad);
            if (bad) break;
            if (has_next) load_op(0, tn);  // the x MMAs and corr_x are done with the x rows
            // ---- y
            if (tid == 0) issue(sth, stl, MRY, 1, C::T2, nks, &bars[2]);
            corr_y();
            // the y epilogue overwrites the y MMAs' own operand (T) in place: all of them must be done
            if (!mbar_wait(&bars[2], ph, kWaitNs)) bad = 1;
            if (!mbar_wait(&bars[3], ph, kWaitNs)) bad = 1;
            tmem_fence_after_sync();
            epi(std::integral_constant<int, S2>{}, MR, 0, C::T2, [](int ap, int bp) { return ap + S3 * bp; });
            tmem_fence_before_sync();
            cp_async_wait_all();
            fence_proxy_async_smem();
            bad = __syncthreads_or(bad);
            if (bad) break;
            if (has_next) load_op(1, tn);
            // ---- z
            if (tid == 0) issue(sth, stl, MR, 2, C::T3, nks, &bars[4]);
            corr_z();
            if (!mbar_wait(&bars[4], ph, kWaitNs)) bad = 1;
            tmem_fence_after_sync();
            epi_z(0, (C::T3 + 1) / 2);
            if (!mbar_wait(&bars[5], ph, kWaitNs)) bad = 1;
            tmem_fence_after_sync();
            epi_z((C::T3 + 1) / 2, C::T3);
            ph ^= 1u;
            tmem_fence_before_sync();
            cp_async_wait_all();
            fence_proxy_async_smem();
            bad = __syncthreads_or(bad);
            ++ntrip;
            if (bad) break;
            if (has_next) load_op(2, tn);
        }
    }
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    double n2 = 0.0, w2 = 0.0;
    if (!bad) {
        double* cs = reinterpret_cast<double*>(xh);  // the operand images are no longer read
        if (!root && tid < KK) {
#pragma unroll
            for (int q = 0; q < K; ++q) cs[tid * K + q] = corr[q];
        }
        __syncthreads();
        double* dst = ch.slot < 0 ? TR.ocoef + (size_t)it.node * BS : partials + (size_t)ch.slot * BS;
        for (int t = 0; t < C::T3; ++t) {
            uint32_t a[2 * K];
            tmem_span_ld<0, 2 * K>(tlane + (uint32_t)(C::COL_ACC + ACCW * t + 2 * K * half), a);
            tmem_span_wait<0, 2 * K>(a);
            const int m = 128 * t + 32 * quarter + lane;
            const int ap = m % S3, bp = m / S3;
            if (ap < K2 && bp < K2) {
#pragma unroll
                for (int cc = 0; cc < K; ++cc) {
                    const int c = K * half + cc;
                    double v = (double)__uint_as_float(a[2 * cc]) + (double)__uint_as_float(a[2 * cc + 1]);
                    const bool sss = ap < K && bp < K && c < K;
                    if (!root && sss) v -= cs[(ap + K * bp) * K + c];
                    dst[ap + K2 * (bp + K2 * c)] = v;
                    n2 += v * v;
                    if (!sss) w2 += v * v;
                }
            }
        }
    }
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    if (warp == 0) tmem_dealloc(tbase, C::TCOLS);
    if (bad) {
        if (tid == 0) atomicExch(err_out, 1);
        return;
    }
    double* red = reinterpret_cast<double*>(xh + 8 * KKK);
    block_sum2(n2, w2, red);
    if (tid == 0) {
        if (ch.slot < 0) {
            TR.onorm2[it.node] = n2;
            TR.ownorm2[it.node] = w2;
        }
        atomicAdd(ntrip_out, ntrip);
    }
}

}  // namespace mwb
