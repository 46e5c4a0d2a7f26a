// mw_slice.hpp -- BF16 fixed-point slices of FP64 rows, and the shared-memory image layouts of the
// tensor-core x step (k_happly).  Shared by the host (operator images) and the device (block images).
//
// A row v[0 .. n) with largest magnitude m = f 2^e (f in [1/2, 1)) is written as
//     v = 2^e (n1 2^-8 + n2 2^-16 + n3 2^-24 [+ n4 2^-32]) + r,
// with integers |n1| <= 256, |n2|, |n3|, |n4| <= 128 (each slice rounded to nearest from what the previous
// ones leave): |r| <= 2^(e-25) with three slices (operators), 2^(e-33) with four (data blocks).  Every
// slice value n 2^(e - 8 s) has at most 8 significant bits, so it is exact in BF16.  Products of a data
// slice and an operator slice are then exact multiples of one quantum per (row, column, slice pair), and
// sums of up to 2^5 of them stay below 2^24 quanta: the tensor core's FP32 accumulation adds them without
// rounding.  This is the splitting idea of the Ozaki scheme (Ozaki, Ogita, Oishi & Rump, Numer.
// Algorithms 59, 2012; on integer/low-precision matrix engines: Ootomo, Ozaki & Yokota, IJHPCA 2024) with
// per-row power-of-two scales.  The data side takes a fourth slice because a data block's slicing error
// is the same in every triple that reads the block (it does not average out over the operator's terms),
// while the remainder relative to the row maximum is coarse for the small entries of a row.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#ifdef __CUDACC__
#define MWB_HD __host__ __device__
#else
#define MWB_HD
#endif

namespace mwb {

// the three slices of each value of a row (FP32 values, each exactly representable in BF16)
MWB_HD inline void slice3_row(const double* v, int n, int stride, float* s0, float* s1, float* s2) {
    double m = 0.0;
    for (int i = 0; i < n; ++i) m = fmax(m, fabs(v[i * stride]));
    int e = 0;
    if (m > 0.0) frexp(m, &e);
    for (int i = 0; i < n; ++i) {
        const double u = ldexp(v[i * stride], -e);  // |u| < 1
        const double a = rint(u * 256.0);
        double r = u - a * (1.0 / 256.0);  // exact
        const double b = rint(r * 65536.0);
        r -= b * (1.0 / 65536.0);  // exact
        const double c = rint(r * 16777216.0);
        s0[i] = (float)ldexp(a, e - 8);
        s1[i] = (float)ldexp(b, e - 16);
        s2[i] = (float)ldexp(c, e - 24);
    }
}

// Four slices of one value with the remainder after the first slice carried in FP32: r1 = u - s0
// (|r1| <= 2^-9 |m|) is exact in FP64 and rounded to FP32 once (2^-33 of the row maximum, the size of the
// last slice's half quantum); the later remainders are exact in FP32.  One FP64 multiply, rounding and FMA
// per value; the first three slices equal slice3_row's except where r1 rounds at that level.
MWB_HD inline void slice4_value(double v, double scale, float inv256, float& s0, float& s1, float& s2, float& s3) {
    const double u = v * scale;  // |u| < 1, exact (power-of-two scale)
    const double a = rint(u * 256.0);
    const float r1 = (float)fma(a, -1.0 / 256.0, u);
    const float b = rintf(r1 * 65536.0f);
    const float r2 = fmaf(b, -1.0f / 65536.0f, r1);
    const float c = rintf(r2 * 16777216.0f);
    const float r3 = fmaf(c, -1.0f / 16777216.0f, r2);
    const float d = rintf(r3 * 4294967296.0f);
    s0 = (float)a * inv256;
    s1 = b * (inv256 * (1.0f / 256.0f));
    s2 = c * (inv256 * (1.0f / 65536.0f));
    s3 = d * (inv256 * (1.0f / 16777216.0f));
}

// BF16 bits of a float with at most 8 significant bits (the low 16 bits of its pattern are zero)
MWB_HD inline uint16_t bf16_bits_exact(float x) {
    uint32_t u;
#ifdef __CUDA_ARCH__
    u = __float_as_uint(x);
#else
    std::memcpy(&u, &x, 4);
#endif
    return (uint16_t)(u >> 16);
}

// Image geometry of the tensor-core x step for 2k = K2 <= 20 (see k_happly).  A "chunk" is R rows x 16
// bytes (8 BF16 values per row); row r = y + K2 z of the data.
//   data block image: slices 0, 1, 2, 3, each NCHM chunks holding x = 0 .. 8 NCHM - 1 (zero for x >= K2);
//   then, when K2 > 16, two packed chunks holding per row [s0 | s1 | s2 | s3] of x = 16 .. K2 - 1
//   (LO = K2 - 16 <= 4 values per slice), so that one 16-deep MMA step covers the rest of x for all slices;
//   operator image, one per NS matrix M[x'][x]: (a) for each data slice q = 0, 1, 2 an operand of
//   NBQ = NCOL + NCOL2 rows x NCHM chunks: row b W + x' (column block b = 0, 1, 2 of the whole matrix)
//   holds slice b - q of M[x'][0 .. 8 NCHM) when b >= q, and row NCOL + b W2 + x' (x' < k) holds slice
//   b - q of the s->s block row M[x'][0 .. k), zero elsewhere (slice pairs of equal weight land in equal
//   output columns); data slice 3 takes the operand of slice 2 (column block 2 = operator slice 0, the
//   products of weight 2^-40 added into block 2); (b) when K2 > 16, the packed step's operand, two chunks
//   of NCOL rows: row b W + x' holds, at K offset 4 q (q = 0, 1, 2), slice b - q of M[x'][16 ..] when
//   b >= q, and row 2 W + x' at K offset 12 (data slice 3) slice 0, zero elsewhere.
struct XGeo {
    int K2, R, TILES, NCHM, PACK, LO, W, NCOL, W2, NCOL2, NBQ, IMGB, OPB_Q, OPB_A, OPB_B, OPB;
    MWB_HD explicit XGeo(int k2)
        : K2(k2), R(k2 * k2), TILES((k2 * k2 + 127) / 128), NCHM(k2 > 8 ? 2 : 1), PACK(k2 > 16 ? 1 : 0),
          LO(k2 > 16 ? k2 - 16 : 0), W(k2), NCOL((3 * k2 + 15) / 16 * 16), W2(k2 / 2),
          NCOL2((3 * (k2 / 2) + 15) / 16 * 16),
          NBQ((3 * k2 + 15) / 16 * 16 + (3 * (k2 / 2) + 15) / 16 * 16),
          IMGB((4 * (k2 > 8 ? 2 : 1) + (k2 > 16 ? 2 : 0)) * k2 * k2 * 16),
          OPB_Q((k2 > 8 ? 2 : 1) * ((3 * k2 + 15) / 16 * 16 + (3 * (k2 / 2) + 15) / 16 * 16) * 16),
          OPB_A(3 * (k2 > 8 ? 2 : 1) * ((3 * k2 + 15) / 16 * 16 + (3 * (k2 / 2) + 15) / 16 * 16) * 16),
          OPB_B(k2 > 16 ? 2 * ((3 * k2 + 15) / 16 * 16) * 16 : 0),
          OPB(3 * (k2 > 8 ? 2 : 1) * ((3 * k2 + 15) / 16 * 16 + (3 * (k2 / 2) + 15) / 16 * 16) * 16 +
              (k2 > 16 ? 2 * ((3 * k2 + 15) / 16 * 16) * 16 : 0)) {}
};

// Split column layout of the CUDA-core GEMM tiles (tile width NT in {4, 5}): column n of a row is stored
// at 4 (n / NT) + n % NT when n % NT < 4, else at 4 NTILES + n / NT, so that a tile's first four values
// are one 16-byte load and the fifth values of consecutive tiles are contiguous.
MWB_HD inline int split_pos(int n, int nt, int ntiles) {
    const int t = n / nt, j = n - t * nt;
    return j < 4 ? 4 * t + j : 4 * ntiles + t;
}

}  // namespace mwb
