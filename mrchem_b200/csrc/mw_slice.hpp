// mw_slice.hpp -- three-slice BF16 fixed-point form of FP64 rows, and the shared-memory image layouts of
// the tensor-core x step (k_happly).  Shared by the host (operator images) and the device (block images).
//
// A row v[0 .. n) with largest magnitude m = f 2^e (f in [1/2, 1)) is written as
//     v = 2^e (n1 2^-8 + n2 2^-16 + n3 2^-24) + r,   |r| <= 2^(e-25),
// with integers |n1| <= 256, |n2|, |n3| <= 128 (each slice rounded to nearest from what the previous
// ones leave).  Every slice value n 2^(e - 8 s) has at most 8 significant bits, so it is exact in BF16.
// Products of a data slice and an operator slice are then exact multiples of one quantum per
// (row, column, slice pair), and sums of up to 2^5 of them stay below 2^24 quanta: the tensor core's FP32
// accumulation adds them without rounding.  This is the splitting idea of the Ozaki scheme (Ozaki,
// Ogita, Oishi & Rump, Numer. Algorithms 59, 2012; on integer/low-precision matrix engines: Ootomo,
// Ozaki & Yokota, IJHPCA 2024) with per-row power-of-two scales.
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

// Image geometry of the tensor-core x step for 2k = K2 (see k_happly):
//   data block image: 3 slices, each NCH chunks of R rows x 16 bytes (row r = y + K2 z holds x = 8c ..
//   8c + 7 of chunk c, BF16, zero for x >= K2);
//   operator image: (a) the whole NS matrix, 2 KSTEPS chunks of NB rows x 16 bytes, rows [2W, 3W) /
//   [3W, 4W) / [4W, 5W) = slices 0 / 1 / 2 of M[x'][.], all other rows zero; then (b) its top-left
//   k x k block (the s->s part, x', x < k), 2 chunks of NB2 rows, rows [2W2, 3W2) / [3W2, 4W2) /
//   [4W2, 5W2) = slices of M[x'][0 .. k) (W2 = k).
struct XGeo {
    int K2, R, TILES, NCH, KSTEPS, W, NCOL, NB, SLICE, IMGB, W2, NCOL2, NB2, OPB_MAIN, OPB;
    MWB_HD explicit XGeo(int k2)
        : K2(k2), R(k2 * k2), TILES((k2 * k2 + 127) / 128), NCH((k2 + 7) / 8), KSTEPS(((k2 + 7) / 8 + 1) / 2), W(k2),
          NCOL((3 * k2 + 15) / 16 * 16), NB(2 * k2 + (3 * k2 + 15) / 16 * 16), SLICE(((k2 + 7) / 8) * k2 * k2 * 16),
          IMGB(3 * ((k2 + 7) / 8) * k2 * k2 * 16), W2(k2 / 2), NCOL2((3 * (k2 / 2) + 15) / 16 * 16),
          NB2(k2 + (3 * (k2 / 2) + 15) / 16 * 16),
          OPB_MAIN(2 * (((k2 + 7) / 8 + 1) / 2) * (2 * k2 + (3 * k2 + 15) / 16 * 16) * 16),
          OPB(2 * (((k2 + 7) / 8 + 1) / 2) * (2 * k2 + (3 * k2 + 15) / 16 * 16) * 16 +
              2 * (k2 + (3 * (k2 / 2) + 15) / 16 * 16) * 16) {}
};

// Split column layout of the CUDA-core GEMM tiles (tile width NT in {4, 5}): column n of a row is stored
// at 4 (n / NT) + n % NT when n % NT < 4, else at 4 NTILES + n / NT, so that a tile's first four values
// are one 16-byte load and the fifth values of consecutive tiles are contiguous.
MWB_HD inline int split_pos(int n, int nt, int ntiles) {
    const int t = n / nt, j = n - t * nt;
    return j < 4 ? 4 * t + j : 4 * ntiles + t;
}

}  // namespace mwb
