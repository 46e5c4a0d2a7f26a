// mw_math.hpp -- host-side set-up mathematics of the MW apply: quadrature, scaling bases, two-scale
// filters, separated Gaussian expansion of the kernels and the non-standard-form (NS) 1-D operator
// tables that the device kernels read.
//
// Published methods restated here (MRCPP, which the reference calls for this, is not vendored):
//   Alpert 1993 / Alpert, Beylkin, Gines & Vozovoi 2002 (bases, filters);
//   Beylkin, Coifman & Rokhlin 1991 (NS form);
//   Harrison, Fann, Yanai, Gan & Beylkin 2004 and Beylkin & Monzon 2005 (Gaussian expansion of
//   1/r and exp(-mu r)/r by the trapezoidal rule in s = log t).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace mwb {

// FP32 -> TF32 (10 explicit mantissa bits) rounded to nearest with ties away from zero, the rounding
// of the device's TF32 split; infinities and NaNs pass unchanged
inline float tf32_round(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}


constexpr double kPi = 3.14159265358979323846;

// Gauss-Legendre rule on [0,1], ascending nodes.
inline void gl01(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    auto legendre_pair = [n](double z, double& pn, double& pn1) {
        double p0 = 1.0, p1 = z;
        if (n == 0) { pn = 1.0; pn1 = 0.0; return; }
        for (int j = 2; j <= n; ++j) {
            double p2 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p0) / j;
            p0 = p1;
            p1 = p2;
        }
        pn = p1;
        pn1 = p0;
    };
    for (int i = 0; i < n; ++i) {
        double z = std::cos(kPi * (i + 0.75) / (n + 0.5));
        for (int it = 0; it < 100; ++it) {
            double pn, pn1;
            legendre_pair(z, pn, pn1);
            double dp = n * (z * pn - pn1) / (z * z - 1.0);
            double dz = pn / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        double pn, pn1;
        legendre_pair(z, pn, pn1);
        double dp = n * (z * pn - pn1) / (z * z - 1.0);
        x[n - 1 - i] = 0.5 * (z + 1.0);
        w[n - 1 - i] = 1.0 / ((1.0 - z * z) * dp * dp);
    }
}

// Orthonormal shifted Legendre values sqrt(2p+1) P_p(2t-1), p < np.
inline void leg01(double t, int np, double* out) {
    double z = 2.0 * t - 1.0, p0 = 1.0, p1 = z;
    if (np > 0) out[0] = 1.0;
    if (np > 1) out[1] = std::sqrt(3.0) * z;
    for (int p = 2; p < np; ++p) {
        double p2 = ((2.0 * p - 1.0) * z * p1 - (p - 1.0) * p0) / p;
        p0 = p1;
        p1 = p2;
        out[p] = std::sqrt(2.0 * p + 1.0) * p2;
    }
}

// d/dt of the normalised shifted Legendre polynomials Pt_p(t) = sqrt(2p+1) P_p(2t - 1) on [0,1],
// from P'_{p+1} = P'_{p-1} + (2p + 1) P_p
inline void leg01_deriv(double t, int np, double* out) {
    const double z = 2.0 * t - 1.0;
    std::vector<double> P(np + 1), dP(np + 1, 0.0);
    P[0] = 1.0;
    if (np > 0) P[1] = z;
    for (int p = 1; p < np; ++p) P[p + 1] = ((2.0 * p + 1.0) * z * P[p] - p * P[p - 1]) / (p + 1.0);
    if (np > 1) dP[1] = 1.0;
    for (int p = 1; p + 1 < np; ++p) dP[p + 1] = dP[p - 1] + (2.0 * p + 1.0) * P[p];
    for (int p = 0; p < np; ++p) out[p] = 2.0 * std::sqrt(2.0 * p + 1.0) * dP[p];
}

struct ScalingBasis {
    int type = 0;  // 0 interpolating (Gauss-Legendre nodes), 1 Legendre
    int k = 0;
    std::vector<double> qx, qw;
    std::vector<double> lq;  // lq[j*k+i] = Pt_i(qx[j]) (interpolating expansion)

    void init(int type_, int order) {
        type = type_;
        k = order + 1;
        gl01(k, qx, qw);
        lq.assign(k * k, 0.0);
        for (int j = 0; j < k; ++j) leg01(qx[j], k, &lq[j * k]);
    }
    // all k scaling functions at x in [0,1]
    void values(double x, double* out) const {
        std::vector<double> L(k);
        leg01(x, k, L.data());
        if (type == 1) {
            for (int j = 0; j < k; ++j) out[j] = L[j];
            return;
        }
        for (int j = 0; j < k; ++j) {
            double v = 0.0;
            for (int i = 0; i < k; ++i) v += lq[j * k + i] * L[i];
            out[j] = v * std::sqrt(qw[j]);
        }
    }
    // first derivatives of all k scaling functions at x in [0,1]
    void derivs(double x, double* out) const {
        std::vector<double> L(k);
        leg01_deriv(x, k, L.data());
        if (type == 1) {
            for (int j = 0; j < k; ++j) out[j] = L[j];
            return;
        }
        for (int j = 0; j < k; ++j) {
            double v = 0.0;
            for (int i = 0; i < k; ++i) v += lq[j * k + i] * L[i];
            out[j] = v * std::sqrt(qw[j]);
        }
    }
};

// Unit-scale blocks of the first-derivative operator with numerical flux parameters (a, b)
// (Alpert, Beylkin, Gines & Vozovoi 2002).  On a cell, integrating phi_i f' by parts with the value
// of f at the right interface taken as (1-a) f_left + a f_right and at the left interface as
// b f_left + (1-b) f_right gives, for output cell l and input cell l - delta:
//   T(0)[i][j]  = (1-a) phi_i(1) phi_j(1) - (1-b) phi_i(0) phi_j(0) - int phi_i' phi_j
//   T(-1)[i][j] = a phi_i(1) phi_j(0)        (input cell l + 1)
//   T(+1)[i][j] = -b phi_i(0) phi_j(1)       (input cell l - 1)
// a = b = 0: the cell-local derivative; a = b = 1/2: the central flux.  At scale n the blocks scale
// with 2^n.  T[delta + 1] holds T(delta), k x k row-major.
inline void derivative_blocks(const ScalingBasis& B, double a, double b, std::vector<double> T[3]) {
    const int k = B.k;
    std::vector<double> p0(k), p1(k), dq(k), pq(k);
    B.values(0.0, p0.data());
    B.values(1.0, p1.data());
    for (int d = 0; d < 3; ++d) T[d].assign((size_t)k * k, 0.0);
    std::vector<double> I(k * k, 0.0);  // int phi_i' phi_j (k-point rule exact: degree 2k - 3)
    for (int q = 0; q < k; ++q) {
        B.derivs(B.qx[q], dq.data());
        B.values(B.qx[q], pq.data());
        for (int i = 0; i < k; ++i)
            for (int j = 0; j < k; ++j) I[i * k + j] += B.qw[q] * dq[i] * pq[j];
    }
    for (int i = 0; i < k; ++i)
        for (int j = 0; j < k; ++j) {
            T[1][i * k + j] = (1.0 - a) * p1[i] * p1[j] - (1.0 - b) * p0[i] * p0[j] - I[i * k + j];
            T[0][i * k + j] = a * p1[i] * p0[j];
            T[2][i * k + j] = -b * p0[i] * p1[j];
        }
}

// Two-scale filter F = [[H0 H1];[G0 G1]] (2k x 2k, row-major).  H by exact 2k-point quadrature;
// G rows: orthonormal complement built from [e_j, -e_j]/sqrt2 by twice-repeated Gram-Schmidt.
inline std::vector<double> two_scale_filter(const ScalingBasis& B) {
    const int k = B.k, K2 = 2 * k;
    std::vector<double> F(K2 * K2, 0.0), gx, gw, pa(k), pb(k);
    gl01(K2, gx, gw);
    for (int q = 0; q < K2; ++q) {
        B.values(gx[q], pb.data());
        for (int c = 0; c < 2; ++c) {
            B.values(0.5 * (gx[q] + c), pa.data());
            for (int j = 0; j < k; ++j)
                for (int i = 0; i < k; ++i) F[j * K2 + c * k + i] += gw[q] * pa[j] * pb[i] / std::sqrt(2.0);
        }
    }
    for (int j = 0; j < k; ++j) {
        std::vector<double> v(K2, 0.0);
        v[j] = 1.0 / std::sqrt(2.0);
        v[k + j] = -1.0 / std::sqrt(2.0);
        for (int pass = 0; pass < 2; ++pass)
            for (int r = 0; r < k + j; ++r) {
                double d = 0.0;
                for (int a = 0; a < K2; ++a) d += F[r * K2 + a] * v[a];
                for (int a = 0; a < K2; ++a) v[a] -= d * F[r * K2 + a];
            }
        double nv = 0.0;
        for (double e : v) nv += e * e;
        nv = std::sqrt(nv);
        for (int a = 0; a < K2; ++a) F[(k + j) * K2 + a] = v[a] / nv;
    }
    return F;
}

// Quadrature matrix W[j*k+q] = w_q phi_j(x_q): s_j = 2^{-(n)/2} sum_q W[j][q] f(point q) per dim.
inline std::vector<double> quadrature_matrix(const ScalingBasis& B) {
    const int k = B.k;
    std::vector<double> W(k * k), p(k);
    for (int q = 0; q < k; ++q) {
        B.values(B.qx[q], p.data());
        for (int j = 0; j < k; ++j) W[j * k + q] = B.qw[q] * p[j];
    }
    return W;
}

struct GaussTerm {
    double alpha, beta;
};

// Trapezoidal rule in s on 1/r = 2/sqrt(pi) int exp(-r^2 e^{2s} + s) ds (times exp(-mu^2 e^{-2s}/4)
// for exp(-mu r)/r).  Step from the trapezoid error 2 sqrt2 exp(-pi^2/(2h)) <= eps; the range covers
// [r_min, r_max] with tails below eps/10.
inline std::vector<GaussTerm> kernel_expansion(double mu, double eps, double r_min, double r_max) {
    const double h = kPi * kPi / (2.0 * std::log(2.0 * std::sqrt(2.0) / eps));
    const double s_hi = std::log((std::sqrt(-std::log(0.1 * eps)) + 1.0) / r_min);
    double s_lo = std::log(0.1 * eps * std::sqrt(kPi) / (2.0 * r_max));
    if (mu > 0.0) s_lo = std::max(s_lo, 0.5 * std::log(mu * mu / (4.0 * -std::log(1e-3 * eps))));
    const int M = (int)std::ceil((s_hi - s_lo) / h) + 1;
    std::vector<GaussTerm> t(M);
    for (int m = 0; m < M; ++m) {
        double s = s_lo + m * h;
        double beta = 2.0 * h / std::sqrt(kPi) * std::exp(s);
        if (mu > 0.0) beta *= std::exp(-0.25 * mu * mu * std::exp(-2.0 * s));
        t[m] = {std::exp(2.0 * s), beta};
    }
    return t;
}

// Scaling-function operator matrices of the 1-D Gaussian exp(-alpha x^2).
//   T^n(l)_ij = 2^{-n} int_{-1}^{1} C_ij(t) exp(-alpha 4^{-n} (t + l)^2) dt,
//   C_ij(t) = int phi_i(u) phi_j(u - t) du  (cross-correlation, a polynomial on each half),
// expanded in shifted Legendre polynomials on each half so that T needs only Gaussian moments.
class GaussianOperatorBuilder {
public:
    GaussianOperatorBuilder(const ScalingBasis& B, const std::vector<double>& F) : B_(B), F_(F) {
        k_ = B.k;
        const int K2 = 2 * k_;
        std::vector<double> tx, tw, P(K2), pu(k_), pv(k_);
        gl01(K2, tx, tw);
        cpos_.assign((size_t)k_ * k_ * K2, 0.0);
        cneg_.assign((size_t)k_ * k_ * K2, 0.0);
        for (int q = 0; q < K2; ++q) {
            const double t = tx[q];
            leg01(t, K2, P.data());
            for (int r = 0; r < k_; ++r) {
                double u = t + (1.0 - t) * B.qx[r], wu = (1.0 - t) * B.qw[r];
                B.values(u, pu.data());
                B.values(u - t, pv.data());
                for (int i = 0; i < k_; ++i)
                    for (int j = 0; j < k_; ++j) {
                        double c = tw[q] * wu * pu[i] * pv[j];
                        for (int p = 0; p < K2; ++p) cpos_[((size_t)i * k_ + j) * K2 + p] += c * P[p];
                    }
                double u2 = t * B.qx[r], wu2 = t * B.qw[r];
                B.values(u2, pu.data());
                B.values(u2 - t + 1.0, pv.data());
                for (int i = 0; i < k_; ++i)
                    for (int j = 0; j < k_; ++j) {
                        double c = tw[q] * wu2 * pu[i] * pv[j];
                        for (int p = 0; p < K2; ++p) cneg_[((size_t)i * k_ + j) * K2 + p] += c * P[p];
                    }
            }
        }
        gl01(K2 + 20, px_, pw_);
    }

    // int_0^1 Pt_p(t) exp(-a (t - c)^2) dt for p < 2k; panels graded away from the point of
    // [0,1] closest to c, with the unit min(a^{-1/2}, 1/(2 a dist)).
    void moments(double a, double c, double* m) const {
        const int np = 2 * k_;
        for (int p = 0; p < np; ++p) m[p] = 0.0;
        const double cs = std::min(std::max(c, 0.0), 1.0), dist = std::fabs(c - cs);
        if (a * dist * dist > 800.0) return;
        std::vector<double> bp;
        if (a <= 4.0) {
            bp = {0.0, 1.0};
        } else {
            double u = 1.0 / std::sqrt(a);
            if (dist > 0.0) u = std::min(u, 1.0 / (2.0 * a * dist));
            std::vector<double> lo_side, hi_side;
            for (double s = 0.0;; s = (s == 0.0 ? 1.0 : 2.0 * s)) {
                double b = cs + s * u;
                if (b >= 1.0) { hi_side.push_back(1.0); break; }
                hi_side.push_back(b);
                if (a * (b - c) * (b - c) > 800.0) break;
            }
            for (double s = 0.0;; s = (s == 0.0 ? 1.0 : 2.0 * s)) {
                double b = cs - s * u;
                if (b <= 0.0) { lo_side.push_back(0.0); break; }
                lo_side.push_back(b);
                if (a * (b - c) * (b - c) > 800.0) break;
            }
            for (size_t i = lo_side.size(); i-- > 1;) bp.push_back(lo_side[i]);
            for (double b : hi_side) bp.push_back(b);
        }
        std::vector<double> P(np);
        for (size_t i = 0; i + 1 < bp.size(); ++i) {
            const double lo = bp[i], hi = bp[i + 1];
            if (hi <= lo) continue;
            for (size_t q = 0; q < px_.size(); ++q) {
                double t = lo + (hi - lo) * px_[q];
                double g = (hi - lo) * pw_[q] * std::exp(-a * (t - c) * (t - c));
                leg01(t, np, P.data());
                for (int p = 0; p < np; ++p) m[p] += g * P[p];
            }
        }
    }

    // T^n(l) (k x k, row-major) for exp(-alpha x^2)
    void scaling(double alpha, int n, long l, double* T) const {
        const int K2 = 2 * k_;
        const double a = alpha * std::ldexp(1.0, -2 * n);
        std::vector<double> mp(K2), mm(K2);
        moments(a, -(double)l, mp.data());
        moments(a, 1.0 - (double)l, mm.data());
        const double fac = std::ldexp(1.0, -n);
        for (int i = 0; i < k_; ++i)
            for (int j = 0; j < k_; ++j) {
                const double* cp = &cpos_[((size_t)i * k_ + j) * K2];
                const double* cm = &cneg_[((size_t)i * k_ + j) * K2];
                double s = 0.0;
                for (int p = 0; p < K2; ++p) s += cp[p] * mp[p] + cm[p] * mm[p];
                T[i * k_ + j] = fac * s;
            }
    }

    // NS matrix at scale n, offset l (2k x 2k; rows = output s|d, cols = input s|d):
    //   NS = F [[T(2l) T(2l-1)];[T(2l+1) T(2l)]]_{n+1} F^T
    void ns(double alpha, int n, long l, double* NS, std::vector<std::pair<long, std::vector<double>>>& cache) const {
        const int K2 = 2 * k_;
        auto get = [&](long lp) -> const double* {
            for (auto& e : cache)
                if (e.first == lp) return e.second.data();
            std::vector<double> T(k_ * k_);
            scaling(alpha, n + 1, lp, T.data());
            cache.emplace_back(lp, std::move(T));
            return cache.back().second.data();
        };
        std::vector<double> mid(K2 * K2), tmp(K2 * K2);
        for (int co = 0; co < 2; ++co)
            for (int ci = 0; ci < 2; ++ci) {
                const double* T = get(2 * l + co - ci);
                for (int i = 0; i < k_; ++i)
                    for (int j = 0; j < k_; ++j) mid[(co * k_ + i) * K2 + ci * k_ + j] = T[i * k_ + j];
            }
        for (int a = 0; a < K2; ++a)
            for (int b = 0; b < K2; ++b) {
                double s = 0.0;
                for (int c = 0; c < K2; ++c) s += F_[a * K2 + c] * mid[c * K2 + b];
                tmp[a * K2 + b] = s;
            }
        for (int a = 0; a < K2; ++a)
            for (int b = 0; b < K2; ++b) {
                double s = 0.0;
                for (int c = 0; c < K2; ++c) s += tmp[a * K2 + c] * F_[b * K2 + c];
                NS[a * K2 + b] = s;
            }
    }
    int k() const { return k_; }

private:
    const ScalingBasis& B_;
    std::vector<double> F_;
    int k_ = 0;
    std::vector<double> cpos_, cneg_, px_, pw_;
};

}  // namespace mwb
