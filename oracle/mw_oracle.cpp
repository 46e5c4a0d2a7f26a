// mw_oracle.cpp -- FP64 CPU restatement of the multiwavelet (MW) operator apply.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle for the B200 path: only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.  The product library
// (mrchem_b200/csrc) never links or calls it.
//
// The reference (MRChem) calls MRCPP for this path, and MRCPP is an un-vendored submodule
// (.gitmodules:4-6, external/mrcpp/ is empty; revision bd40f63 per
// tests/h2_scf_hf/reference/mrchem.stdout:26).  Its source is therefore not available and this is a
// restatement of the published method, not of MRCPP's code:
//   * scaling bases: Alpert 1993 (Legendre) and Alpert, Beylkin, Gines & Vozovoi 2002
//     (interpolating, Gauss-Legendre nodes); two-scale filters by exact Gauss-Legendre quadrature;
//   * non-standard (NS) form of an operator: Beylkin, Coifman & Rokhlin 1991;
//   * separated Gaussian expansion of 1/r and exp(-mu r)/r: trapezoidal discretisation of
//     1/r = 2/sqrt(pi) int exp(-r^2 e^{2s} + s) ds (Harrison, Fann, Yanai, Gan & Beylkin 2004;
//     Beylkin & Monzon 2005);
//   * adaptive NS-form apply with wavelet-norm refinement of the output tree and operator-norm
//     screening: Frediani, Fossgaard, Flaa & Ruud 2013.
// The call contract follows the reference's call sites:
//   mrcpp::apply(prec, out, op, inp)   src/scf_solver/HelmholtzVector.cpp:176,
//                                      src/qmoperators/two_electron/CoulombPotential.cpp:85
//   PoissonOperator(MRA, prec)         src/SCFDriver.cpp:279
//   HelmholtzOperator(MRA, mu, prec)   src/scf_solver/HelmholtzVector.cpp:171
//   MultiResolutionAnalysis(world, basis, max_depth)  src/mrenv.cpp:52,64-72
//
// Layout conventions (shared with the product, by design, so results can be compared):
//   * a node at depth d (scale n = n0 + d) has translation t (per dim, t >= 0, relative to the
//     world corner: box lower corner = corner * 2^-n0 + t * 2^-n);
//   * a node block holds 8 k^3 doubles as a (2k)^3 tensor, x fastest; index a = c*k + i per dim,
//     where c = 0/1 selects scaling/wavelet (compressed form) or child 0/1 (reconstructed form).
#include <algorithm>
#include <array>
#include <tuple>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------------------------------------
// Quadrature and polynomials
// ---------------------------------------------------------------------------------------------

// Gauss-Legendre nodes and weights on [0,1] (Newton iteration on P_n).
void gauss_legendre01(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int i = 0; i < n; ++i) {
        double z = std::cos(kPi * (i + 0.75) / (n + 0.5));
        double dp = 1.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = z;
            for (int j = 2; j <= n; ++j) {
                double p2 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p0) / j;
                p0 = p1;
                p1 = p2;
            }
            if (n == 1) { p0 = 1.0; p1 = z; }
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        {
            double p0 = 1.0, p1 = z;
            for (int j = 2; j <= n; ++j) {
                double p2 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p0) / j;
                p0 = p1;
                p1 = p2;
            }
            if (n == 1) { p0 = 1.0; p1 = z; }
            dp = n * (z * p1 - p0) / (z * z - 1.0);
        }
        // z runs from +1 to -1 with i; map to ascending nodes on [0,1]
        x[n - 1 - i] = 0.5 * (z + 1.0);
        w[n - 1 - i] = 1.0 / ((1.0 - z * z) * dp * dp);  // 2/((1-z^2)P'^2) halved for [0,1]
    }
}

// d/dt Pt_p(t) for p < np, from (1 - z^2) P_p'(z) = p (P_{p-1}(z) - z P_p(z)) away from the ends and
// P_p'(+-1) = (+-1)^{p+1} p (p + 1) / 2 at them
inline void legendre01_deriv(double t, int np, double* out) {
    const double z = 2.0 * t - 1.0;
    std::vector<double> P(np + 1);
    P[0] = 1.0;
    if (np > 0) P[1] = z;
    for (int p = 1; p < np; ++p) P[p + 1] = ((2.0 * p + 1.0) * z * P[p] - p * P[p - 1]) / (p + 1.0);
    for (int p = 0; p < np; ++p) {
        double d;
        if (p == 0) d = 0.0;
        else if (std::fabs(1.0 - z * z) < 1e-12) d = (z > 0 ? 1.0 : ((p + 1) % 2 == 0 ? 1.0 : -1.0)) * 0.5 * p * (p + 1.0);
        else d = p * (P[p - 1] - z * P[p]) / (1.0 - z * z);
        out[p] = 2.0 * std::sqrt(2.0 * p + 1.0) * d;
    }
}

// Orthonormal shifted Legendre polynomials Pt_p(t) = sqrt(2p+1) P_p(2t-1) on [0,1], p < np.
inline void legendre01(double t, int np, double* out) {
    double z = 2.0 * t - 1.0;
    double p0 = 1.0, p1 = z;
    if (np > 0) out[0] = 1.0;
    if (np > 1) out[1] = std::sqrt(3.0) * z;
    for (int p = 2; p < np; ++p) {
        double p2 = ((2.0 * p - 1.0) * z * p1 - (p - 1.0) * p0) / p;
        p0 = p1;
        p1 = p2;
        out[p] = std::sqrt(2.0 * p + 1.0) * p2;
    }
}

// ---------------------------------------------------------------------------------------------
// Scaling basis and two-scale filters
// ---------------------------------------------------------------------------------------------

struct Basis {
    int type = 0;  // 0 = interpolating, 1 = Legendre
    int k = 0;     // number of scaling functions per dimension = order + 1
    std::vector<double> qx, qw;  // k-point Gauss-Legendre rule on [0,1]
    std::vector<double> F;       // (2k)x(2k): rows [s_0..s_k-1, d_0..d_k-1], cols [child0, child1]

    // phi_j(x) on [0,1]
    double phi(int j, double x) const {
        std::vector<double> L(k);
        legendre01(x, k, L.data());
        if (type == 1) return L[j];
        // interpolating: phi_j = sqrt(w_j) * sum_i Pt_i(x_j) Pt_i(x) (the Lagrange polynomial at
        // node x_j divided by sqrt(w_j))
        std::vector<double> Lj(k);
        legendre01(qx[j], k, Lj.data());
        double v = 0.0;
        for (int i = 0; i < k; ++i) v += Lj[i] * L[i];
        return v * std::sqrt(qw[j]);
    }
    void phi_all(double x, double* out) const {
        for (int j = 0; j < k; ++j) out[j] = phi(j, x);
    }
    // phi_j'(x) on [0,1]
    double dphi(int j, double x) const {
        std::vector<double> L(k);
        legendre01_deriv(x, k, L.data());
        if (type == 1) return L[j];
        std::vector<double> Lj(k);
        legendre01(qx[j], k, Lj.data());
        double v = 0.0;
        for (int i = 0; i < k; ++i) v += Lj[i] * L[i];
        return v * std::sqrt(qw[j]);
    }

    void build(int type_, int order) {
        type = type_;
        k = order + 1;
        gauss_legendre01(k, qx, qw);
        const int K2 = 2 * k;
        F.assign(K2 * K2, 0.0);
        std::vector<double> gx, gw;
        gauss_legendre01(K2, gx, gw);
        // H_c[j][i] = <phi_j, sqrt2 phi_i(2x - c)> = 1/sqrt2 int_0^1 phi_j((u+c)/2) phi_i(u) du
        for (int c = 0; c < 2; ++c) {
            for (int j = 0; j < k; ++j) {
                for (int i = 0; i < k; ++i) {
                    double s = 0.0;
                    for (int q = 0; q < K2; ++q) s += gw[q] * phi(j, 0.5 * (gx[q] + c)) * phi(i, gx[q]);
                    F[j * K2 + c * k + i] = s / std::sqrt(2.0);
                }
            }
        }
        // Wavelet rows: orthonormal complement of the scaling rows.  Candidates are the
        // "difference" vectors [e_j, -e_j]/sqrt2, which never lie in the polynomial space, made
        // orthogonal to it and to each other by two passes of modified Gram-Schmidt.
        for (int j = 0; j < k; ++j) {
            std::vector<double> v(K2, 0.0);
            v[j] = 1.0 / std::sqrt(2.0);
            v[k + j] = -1.0 / std::sqrt(2.0);
            for (int pass = 0; pass < 2; ++pass) {
                for (int r = 0; r < k + j; ++r) {
                    double dot = 0.0;
                    for (int a = 0; a < K2; ++a) dot += F[r * K2 + a] * v[a];
                    for (int a = 0; a < K2; ++a) v[a] -= dot * F[r * K2 + a];
                }
            }
            double nrm = 0.0;
            for (int a = 0; a < K2; ++a) nrm += v[a] * v[a];
            nrm = std::sqrt(nrm);
            for (int a = 0; a < K2; ++a) F[(k + j) * K2 + a] = v[a] / nrm;
        }
    }
};

// ---------------------------------------------------------------------------------------------
// Small tensor kernels.  Tensors are (nx, ny, nz), x fastest.
// ---------------------------------------------------------------------------------------------

// out = M x_dim in, where M is rows x cols with row stride ldm (acts on index along `dim`).
void mode_product(const double* M, int ldm, int rows, int cols, int dim, const double* in, int nx,
                  int ny, int nz, double* out) {
    if (dim == 0) {
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y) {
                const double* src = in + (size_t)nx * (y + (size_t)ny * z);
                double* dst = out + (size_t)rows * (y + (size_t)ny * z);
                for (int a = 0; a < rows; ++a) {
                    double s = 0.0;
                    for (int b = 0; b < cols; ++b) s += M[a * ldm + b] * src[b];
                    dst[a] = s;
                }
            }
    } else if (dim == 1) {
        for (int z = 0; z < nz; ++z)
            for (int a = 0; a < rows; ++a) {
                double* dst = out + (size_t)nx * (a + (size_t)rows * z);
                for (int x = 0; x < nx; ++x) dst[x] = 0.0;
                for (int b = 0; b < cols; ++b) {
                    const double m = M[a * ldm + b];
                    const double* src = in + (size_t)nx * (b + (size_t)ny * z);
                    for (int x = 0; x < nx; ++x) dst[x] += m * src[x];
                }
            }
    } else {
        const size_t plane = (size_t)nx * ny;
        for (int a = 0; a < rows; ++a) {
            double* dst = out + plane * a;
            for (size_t p = 0; p < plane; ++p) dst[p] = 0.0;
            for (int b = 0; b < cols; ++b) {
                const double m = M[a * ldm + b];
                const double* src = in + plane * b;
                for (size_t p = 0; p < plane; ++p) dst[p] += m * src[p];
            }
        }
    }
}

// Apply the same (2k)x(2k) matrix along all three dims of a (2k)^3 tensor (transpose if tr).
void transform3(const std::vector<double>& F, int k, bool tr, const double* in, double* out) {
    const int K2 = 2 * k;
    std::vector<double> M(K2 * K2);
    for (int a = 0; a < K2; ++a)
        for (int b = 0; b < K2; ++b) M[a * K2 + b] = tr ? F[b * K2 + a] : F[a * K2 + b];
    std::vector<double> t1((size_t)K2 * K2 * K2), t2((size_t)K2 * K2 * K2);
    mode_product(M.data(), K2, K2, K2, 0, in, K2, K2, K2, t1.data());
    mode_product(M.data(), K2, K2, K2, 1, t1.data(), K2, K2, K2, t2.data());
    mode_product(M.data(), K2, K2, K2, 2, t2.data(), K2, K2, K2, out);
}

double sq_norm(const double* v, size_t n) {
    double s = 0.0;
    for (size_t i = 0; i < n; ++i) s += v[i] * v[i];
    return s;
}

// squared norm of the wavelet part (all components except the s-s-s sub-cube)
double wavelet_sq_norm(const double* c, int k) {
    const int K2 = 2 * k;
    double s = 0.0;
    for (int z = 0; z < K2; ++z)
        for (int y = 0; y < K2; ++y)
            for (int x = 0; x < K2; ++x) {
                if (x < k && y < k && z < k) continue;
                double v = c[x + K2 * (y + K2 * z)];
                s += v * v;
            }
    return s;
}

// ---------------------------------------------------------------------------------------------
// World (MRA) and trees
// ---------------------------------------------------------------------------------------------

struct MRA {
    int n0 = 0;  // root scale (box edge 2^-n0)
    int corner[3] = {0, 0, 0};
    int boxes[3] = {1, 1, 1};
    int max_depth = 0;
    Basis basis;
    int k() const { return basis.k; }
    size_t bsize() const { return (size_t)8 * basis.k * basis.k * basis.k; }
};

// Collision-free node key: (depth, tx) and (ty, tz), translations < 2^32.
struct Key {
    uint64_t a, b;
    bool operator==(const Key& o) const { return a == o.a && b == o.b; }
};
struct KeyHash {
    size_t operator()(const Key& k) const {
        uint64_t h = k.a * 0x9E3779B97F4A7C15ull ^ (k.b + 0x632BE59BD9B4E019ull + (k.a << 6) + (k.a >> 2));
        return (size_t)(h ^ (h >> 31));
    }
};
inline Key node_key(int depth, const int64_t t[3]) {
    return Key{((uint64_t)depth << 32) | (uint64_t)(uint32_t)t[0],
               ((uint64_t)(uint32_t)t[1] << 32) | (uint64_t)(uint32_t)t[2]};
}

struct Node {
    int depth = 0;
    int64_t t[3] = {0, 0, 0};
    int parent = -1;
    int child0 = -1;  // first of 8 consecutive children, -1 for leaves
    std::vector<double> c;
};

struct Tree {
    const MRA* mra = nullptr;
    std::vector<Node> nodes;
    std::unordered_map<Key, int, KeyHash> index;

    void clear() {
        nodes.clear();
        index.clear();
    }
    int find(int depth, const int64_t t[3]) const {
        auto it = index.find(node_key(depth, t));
        return it == index.end() ? -1 : it->second;
    }
    int add(int depth, const int64_t t[3], int parent) {
        Node nd;
        nd.depth = depth;
        for (int d = 0; d < 3; ++d) nd.t[d] = t[d];
        nd.parent = parent;
        nd.c.assign(mra->bsize(), 0.0);
        nodes.push_back(std::move(nd));
        int id = (int)nodes.size() - 1;
        index[node_key(depth, t)] = id;
        return id;
    }
    void make_roots() {
        clear();
        for (int z = 0; z < mra->boxes[2]; ++z)
            for (int y = 0; y < mra->boxes[1]; ++y)
                for (int x = 0; x < mra->boxes[0]; ++x) {
                    int64_t t[3] = {x, y, z};
                    add(0, t, -1);
                }
    }
    // append the 8 children of node i (child index c = cx + 2cy + 4cz)
    void split(int i) {
        int depth = nodes[i].depth + 1;
        int64_t pt[3] = {nodes[i].t[0], nodes[i].t[1], nodes[i].t[2]};
        int first = (int)nodes.size();
        for (int c = 0; c < 8; ++c) {
            int64_t t[3] = {2 * pt[0] + (c & 1), 2 * pt[1] + ((c >> 1) & 1), 2 * pt[2] + ((c >> 2) & 1)};
            add(depth, t, i);
        }
        nodes[i].child0 = first;
    }
    double square_norm() const {
        double s = 0.0;
        for (const Node& n : nodes)
            if (n.child0 < 0) s += sq_norm(n.c.data(), n.c.size());
        return s;
    }
    // nodes ordered by depth (parents before children)
    std::vector<int> level_order() const {
        std::vector<int> ord(nodes.size());
        for (size_t i = 0; i < ord.size(); ++i) ord[i] = (int)i;
        std::stable_sort(ord.begin(), ord.end(),
                         [&](int a, int b) { return nodes[a].depth < nodes[b].depth; });
        return ord;
    }
    int max_depth_present() const {
        int m = 0;
        for (const Node& n : nodes) m = std::max(m, n.depth);
        return m;
    }
};

// Make every internal node's block the compression of its children's scaling parts
// (bottom-up), so that the leaves alone define the function.
void compress_bottom_up(Tree& tr) {
    const int k = tr.mra->k();
    const int K2 = 2 * k;
    int maxd = tr.max_depth_present();
    std::vector<std::vector<int>> levels(maxd + 1);
    for (size_t i = 0; i < tr.nodes.size(); ++i) levels[tr.nodes[i].depth].push_back((int)i);
    for (int d = maxd - 1; d >= 0; --d) {
        std::vector<int>& lv = levels[d];
#pragma omp parallel for schedule(dynamic, 4)
        for (size_t q = 0; q < lv.size(); ++q) {
            Node& nd = tr.nodes[lv[q]];
            if (nd.child0 < 0) continue;
            std::vector<double> rec((size_t)K2 * K2 * K2);
            for (int c = 0; c < 8; ++c) {
                const Node& ch = tr.nodes[nd.child0 + c];
                int cx = c & 1, cy = (c >> 1) & 1, cz = (c >> 2) & 1;
                for (int z = 0; z < k; ++z)
                    for (int y = 0; y < k; ++y)
                        for (int x = 0; x < k; ++x)
                            rec[(cx * k + x) + K2 * ((cy * k + y) + K2 * (cz * k + z))] =
                                ch.c[x + K2 * (y + K2 * z)];
            }
            transform3(tr.mra->basis.F, k, false, rec.data(), nd.c.data());
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Analytic functions for projection
// ---------------------------------------------------------------------------------------------

// Hydrogen-like orbital, restated from src/analyticfunctions/HydrogenFunction.cpp:28-160
// (radial normalisation constants and polynomials, real solid-harmonic angular parts).
struct Hydrogen {
    int n = 1, l = 0, m = 0;
    double Z = 1.0;
    double o[3] = {0, 0, 0};
    double c0 = 0, c1 = 0, ca = 0;
    void init() {
        double c = 0.0;
        if (n == 1 && l == 0) c = 2.0;
        else if (n == 2 && l == 0) c = 1.0 / (2.0 * std::sqrt(2.0));
        else if (n == 3 && l == 0) c = 1.0 / (9.0 * std::sqrt(3.0));
        else if (n == 2 && l == 1) c = 1.0 / (2.0 * std::sqrt(6.0));
        else if (n == 3 && l == 1) c = 1.0 / (9.0 * std::sqrt(6.0));
        else if (n == 3 && l == 2) c = 1.0 / (9.0 * std::sqrt(30.0));
        c0 = c * std::pow(Z, 1.5);
        c1 = 2.0 * Z / n;
        double a = 0.0;
        if (l == 0) a = 1.0;
        else if (l == 1) a = std::sqrt(3.0);
        else if (l == 2) a = (m <= 2) ? std::sqrt(15.0) : (m == 3 ? std::sqrt(15.0 / 4.0) : std::sqrt(5.0 / 4.0));
        ca = a / (2.0 * std::sqrt(kPi));
    }
    double operator()(const double* r) const {
        double x = r[0] - o[0], y = r[1] - o[1], z = r[2] - o[2];
        double rr = std::sqrt(x * x + y * y + z * z);
        double rho = c1 * rr;
        double poly = 0.0;
        if (n == 1 && l == 0) poly = 1.0;
        else if (n == 2 && l == 0) poly = 2.0 - rho;
        else if (n == 3 && l == 0) poly = 6.0 - 6.0 * rho + rho * rho;
        else if (n == 2 && l == 1) poly = rho;
        else if (n == 3 && l == 1) poly = rho * (4.0 - rho);
        else if (n == 3 && l == 2) poly = rho * rho;
        double radial = c0 * poly * std::exp(-0.5 * rho);
        double ang = 1.0;
        if (l == 1) {
            if (rr == 0.0) return 0.0;
            ang = (m == 0 ? x : (m == 1 ? y : z)) / rr;
        } else if (l == 2) {
            if (rr == 0.0) return 0.0;
            double r2 = rr * rr;
            if (m == 0) ang = x * y / r2;
            else if (m == 1) ang = x * z / r2;
            else if (m == 2) ang = y * z / r2;
            else if (m == 3) ang = (x * x - y * y) / r2;
            else ang = (2.0 * z * z - x * x - y * y) / r2;
        }
        return radial * ca * ang;
    }
};

struct Func {
    // type 1: sum_g c_g (x-X)^px (y-Y)^py (z-Z)^pz exp(-alpha_g |r-R_g|^2)
    struct G { double c, a, R[3]; int p[3]; };
    std::vector<G> gs;
    // type 2: sum_t c_t * A_t(r) * B_t(r) (B absent -> 1)
    struct HP { double c; Hydrogen A, B; bool hasB; };
    std::vector<HP> hs;
    double operator()(const double* r) const {
        double v = 0.0;
        for (const G& g : gs) {
            double dx = r[0] - g.R[0], dy = r[1] - g.R[1], dz = r[2] - g.R[2];
            double e = std::exp(-g.a * (dx * dx + dy * dy + dz * dz));
            double p = 1.0;
            for (int i = 0; i < g.p[0]; ++i) p *= dx;
            for (int i = 0; i < g.p[1]; ++i) p *= dy;
            for (int i = 0; i < g.p[2]; ++i) p *= dz;
            v += g.c * p * e;
        }
        for (const HP& h : hs) v += h.c * h.A(r) * (h.hasB ? h.B(r) : 1.0);
        return v;
    }
};

// Block of node (depth, t) by quadrature: children scaling coefficients at scale n+1 (the
// reconstructed form), then compressed.  Interpolating basis: s_j = 2^{-3(n+1)/2}
// sqrt(w_jx w_jy w_jz) f(node point); Legendre basis: k-point Gauss-Legendre quadrature.
void project_node(const MRA& mra, const Func& f, int depth, const int64_t t[3], double* out) {
    const int k = mra.k();
    const int K2 = 2 * k;
    const int n1 = mra.n0 + depth + 1;
    const double h = std::ldexp(1.0, -n1);  // child box edge
    const double fac = std::pow(2.0, -1.5 * n1);
    const Basis& B = mra.basis;
    std::vector<double> rec((size_t)K2 * K2 * K2);
    std::vector<double> P(k * k);  // P[q*k+j] = phi_j(x_q)
    for (int q = 0; q < k; ++q)
        for (int j = 0; j < k; ++j) P[q * k + j] = B.phi(j, B.qx[q]);
    std::vector<double> fv((size_t)k * k * k);
    for (int c = 0; c < 8; ++c) {
        int cc[3] = {c & 1, (c >> 1) & 1, (c >> 2) & 1};
        double lo[3];
        for (int d = 0; d < 3; ++d)
            lo[d] = mra.corner[d] * std::ldexp(1.0, -mra.n0) + (2 * t[d] + cc[d]) * h;
        for (int z = 0; z < k; ++z)
            for (int y = 0; y < k; ++y)
                for (int x = 0; x < k; ++x) {
                    double r[3] = {lo[0] + h * B.qx[x], lo[1] + h * B.qx[y], lo[2] + h * B.qx[z]};
                    fv[x + k * (y + k * z)] = f(r);
                }
        for (int jz = 0; jz < k; ++jz)
            for (int jy = 0; jy < k; ++jy)
                for (int jx = 0; jx < k; ++jx) {
                    double s;
                    if (B.type == 0) {
                        s = std::sqrt(B.qw[jx] * B.qw[jy] * B.qw[jz]) * fv[jx + k * (jy + k * jz)];
                    } else {
                        s = 0.0;
                        for (int z = 0; z < k; ++z)
                            for (int y = 0; y < k; ++y)
                                for (int x = 0; x < k; ++x)
                                    s += B.qw[x] * B.qw[y] * B.qw[z] * P[x * k + jx] * P[y * k + jy] *
                                         P[z * k + jz] * fv[x + k * (y + k * z)];
                    }
                    rec[(cc[0] * k + jx) + K2 * ((cc[1] * k + jy) + K2 * (cc[2] * k + jz))] = fac * s;
                }
    }
    transform3(B.F, k, false, rec.data(), out);
}

inline double split_threshold(double prec, double ref, int depth) {
    return prec * ref * std::pow(2.0, -0.5 * depth);
}

// Adaptive projection.  Split a node when ||d|| > prec * ||f|| * 2^{-depth/2}, where ||f|| is the
// norm of the current approximation (recomputed after every pass), then compress bottom-up.
void project(Tree& tr, const Func& f, double prec) {
    const MRA& mra = *tr.mra;
    tr.make_roots();
    std::vector<int> work(tr.nodes.size());
    for (size_t i = 0; i < work.size(); ++i) work[i] = (int)i;
    while (!work.empty()) {
#pragma omp parallel for schedule(dynamic, 1)
        for (size_t q = 0; q < work.size(); ++q) {
            Node& nd = tr.nodes[work[q]];
            project_node(mra, f, nd.depth, nd.t, nd.c.data());
        }
        double ref = std::sqrt(tr.square_norm());
        std::vector<int> next;
        for (int i : work) {
            Node& nd = tr.nodes[i];
            if (nd.depth >= mra.max_depth || prec <= 0.0) continue;
            double w = std::sqrt(wavelet_sq_norm(nd.c.data(), mra.k()));
            if (w > split_threshold(prec, ref, nd.depth)) {
                tr.split(i);
                int c0 = tr.nodes[i].child0;
                for (int c = 0; c < 8; ++c) next.push_back(c0 + c);
            }
        }
        work.swap(next);
    }
    compress_bottom_up(tr);
}

// ---------------------------------------------------------------------------------------------
// Convolution operators: separated Gaussian expansion + NS-form 1-D matrices
// ---------------------------------------------------------------------------------------------

// Moments m_p = int_0^1 Pt_p(t) exp(-a (t - c)^2) dt, p < np, by composite Gauss-Legendre
// quadrature on panels graded geometrically away from the point of [0,1] nearest to c.
void gauss_moments(double a, double c, int np, const std::vector<double>& gx,
                   const std::vector<double>& gw, double* m) {
    for (int p = 0; p < np; ++p) m[p] = 0.0;
    const double cs = std::min(std::max(c, 0.0), 1.0);
    const double dist = std::fabs(c - cs);
    if (a * dist * dist > 800.0) return;
    std::vector<double> bps;
    if (a <= 4.0) {
        bps = {0.0, 1.0};
    } else {
        double u = 1.0 / std::sqrt(a);
        if (dist > 0.0) u = std::min(u, 1.0 / (2.0 * a * dist));
        std::vector<double> right, left;
        for (double s = 0.0;; s = (s == 0.0 ? 1.0 : 2.0 * s)) {
            double bp = cs + s * u;
            if (bp >= 1.0) { right.push_back(1.0); break; }
            right.push_back(bp);
            if (a * (bp - c) * (bp - c) > 800.0) break;
        }
        for (double s = 0.0;; s = (s == 0.0 ? 1.0 : 2.0 * s)) {
            double bp = cs - s * u;
            if (bp <= 0.0) { left.push_back(0.0); break; }
            left.push_back(bp);
            if (a * (bp - c) * (bp - c) > 800.0) break;
        }
        for (size_t i = left.size(); i-- > 1;) bps.push_back(left[i]);
        for (double v : right) bps.push_back(v);
    }
    std::vector<double> P(np);
    for (size_t b = 0; b + 1 < bps.size(); ++b) {
        double lo = bps[b], hi = bps[b + 1];
        if (hi <= lo) continue;
        for (size_t q = 0; q < gx.size(); ++q) {
            double t = lo + (hi - lo) * gx[q];
            double g = (hi - lo) * gw[q] * std::exp(-a * (t - c) * (t - c));
            legendre01(t, np, P.data());
            for (int p = 0; p < np; ++p) m[p] += g * P[p];
        }
    }
}

struct Term {
    double alpha, beta;
};

// 1/r ~ sum_m beta_m exp(-alpha_m r^2) on [r_min, r_max] with relative error ~eps, from the
// trapezoidal rule on 1/r = 2/sqrt(pi) int exp(-r^2 e^{2s} + s) ds; for mu > 0 the integrand
// gains the factor exp(-mu^2 e^{-2s}/4), giving exp(-mu r)/r.
std::vector<Term> gauss_expansion(double mu, double eps, double r_min, double r_max) {
    const double h = kPi * kPi / (2.0 * std::log(2.0 * std::sqrt(2.0) / eps));
    const double x_hi = std::sqrt(-std::log(0.1 * eps)) + 1.0;
    const double s_hi = std::log(x_hi / r_min);
    double s_lo = std::log(0.1 * eps * std::sqrt(kPi) / (2.0 * r_max));
    if (mu > 0.0) {
        // exp(-mu^2 e^{-2s}/4) < 1e-3 eps below s_cut
        double s_cut = 0.5 * std::log(mu * mu / (4.0 * -std::log(1e-3 * eps)));
        s_lo = std::max(s_lo, s_cut);
    }
    std::vector<Term> terms;
    int M = (int)std::ceil((s_hi - s_lo) / h) + 1;
    for (int m = 0; m < M; ++m) {
        double s = s_lo + m * h;
        double beta = 2.0 * h / std::sqrt(kPi) * std::exp(s);
        if (mu > 0.0) beta *= std::exp(-0.25 * mu * mu * std::exp(-2.0 * s));
        terms.push_back({std::exp(2.0 * s), beta});
    }
    return terms;
}

// Per (term, depth) band of NS matrices for offsets -L..L.
struct Band {
    bool active = false;
    int L = -1;
    std::vector<double> ns;  // (2L+1) blocks of (2k)^2, offset l at index l+L; NS[aout*2k+ain]
    std::vector<double> t2, x2;  // squared Frobenius norms of the T block and of the rest
};

struct DeltaEntry {
    int d[3];
    double maxb;
    std::vector<std::pair<double, int>> terms;  // (bound, term), sorted by bound descending
};

struct Operator {
    const MRA* mra = nullptr;
    double mu = 0.0;
    double prec = 0.0;
    double eps = 0.0;
    std::vector<Term> terms;
    std::vector<double> cp, cm;  // cross-correlation coefficients [i][j][p] for t>0 and t<0 halves
    std::vector<double> gx, gw;  // panel quadrature rule
    double B0 = 0.0;             // largest root-depth block bound (scale of the operator)
    std::map<int, std::vector<Band>> bands;             // depth -> per-term bands
    std::map<int, std::vector<DeltaEntry>> deltas;      // depth -> offset list
    std::mutex mtx;

    void init(const MRA* m, double mu_, double prec_) {
        mra = m;
        mu = mu_;
        prec = prec_;
        eps = 0.1 * prec;
        const int k = mra->k();
        const int K2 = 2 * k;
        double root_edge = std::ldexp(1.0, -mra->n0);
        double r_max = 0.0;
        for (int d = 0; d < 3; ++d) r_max += std::pow(mra->boxes[d] * root_edge, 2);
        r_max = std::sqrt(r_max);
        double r_min = 0.01 * std::ldexp(root_edge, -mra->max_depth);
        terms = gauss_expansion(mu, eps, r_min, r_max);
        // cross-correlations C_ij(t) = int phi_i(u) phi_j(u - t) du as Legendre series on each half
        const Basis& B = mra->basis;
        std::vector<double> tx, tw;
        gauss_legendre01(K2, tx, tw);
        cp.assign((size_t)k * k * K2, 0.0);
        cm.assign((size_t)k * k * K2, 0.0);
        std::vector<double> P(K2), pu(k), pv(k);
        for (int q = 0; q < K2; ++q) {
            double t = tx[q];
            legendre01(t, K2, P.data());
            std::vector<double> Cp(k * k, 0.0), Cm(k * k, 0.0);
            for (int r = 0; r < k; ++r) {
                // t in [0,1]: u in [t,1], v = u - t
                double u = t + (1.0 - t) * B.qx[r], wu = (1.0 - t) * B.qw[r];
                B.phi_all(u, pu.data());
                B.phi_all(u - t, pv.data());
                for (int i = 0; i < k; ++i)
                    for (int j = 0; j < k; ++j) Cp[i * k + j] += wu * pu[i] * pv[j];
                // tau in [0,1] stands for t = tau - 1: u in [0,tau], v = u - tau + 1
                double u2 = t * B.qx[r], wu2 = t * B.qw[r];
                B.phi_all(u2, pu.data());
                B.phi_all(u2 - t + 1.0, pv.data());
                for (int i = 0; i < k; ++i)
                    for (int j = 0; j < k; ++j) Cm[i * k + j] += wu2 * pu[i] * pv[j];
            }
            for (int i = 0; i < k; ++i)
                for (int j = 0; j < k; ++j)
                    for (int p = 0; p < K2; ++p) {
                        cp[((size_t)i * k + j) * K2 + p] += tw[q] * Cp[i * k + j] * P[p];
                        cm[((size_t)i * k + j) * K2 + p] += tw[q] * Cm[i * k + j] * P[p];
                    }
        }
        gauss_legendre01(K2 + 20, gx, gw);
        // operator scale from the root depth
        std::vector<Band>& b0 = get_bands(0);
        B0 = 0.0;
        for (size_t m = 0; m < terms.size(); ++m) {
            if (!b0[m].active) continue;
            int L = b0[m].L;
            double v = b0[m].t2[L] + b0[m].x2[L];
            B0 = std::max(B0, terms[m].beta * std::pow(v, 1.5));
        }
    }

    // scaling-function matrix T^n(l) for exp(-alpha x^2) at scale n: k x k
    void scaling_matrix(double alpha, int n, long l, double* T) const {
        const int k = mra->k();
        const int K2 = 2 * k;
        double a = alpha * std::ldexp(1.0, -2 * n);
        std::vector<double> mp(K2), mm(K2);
        gauss_moments(a, -(double)l, K2, gx, gw, mp.data());
        gauss_moments(a, 1.0 - (double)l, K2, gx, gw, mm.data());
        double fac = std::ldexp(1.0, -n);
        for (int i = 0; i < k; ++i)
            for (int j = 0; j < k; ++j) {
                double s = 0.0;
                for (int p = 0; p < K2; ++p)
                    s += cp[((size_t)i * k + j) * K2 + p] * mp[p] + cm[((size_t)i * k + j) * K2 + p] * mm[p];
                T[i * k + j] = fac * s;
            }
    }

    // NS matrix at scale n, offset l: F [[T(2l) T(2l-1)];[T(2l+1) T(2l)]]_{n+1} F^T
    void ns_matrix(double alpha, int n, long l, std::map<long, std::vector<double>>& cache,
                   double* NS) const {
        const int k = mra->k();
        const int K2 = 2 * k;
        auto getT = [&](long lp) -> const std::vector<double>& {
            auto it = cache.find(lp);
            if (it != cache.end()) return it->second;
            std::vector<double> T(k * k);
            scaling_matrix(alpha, n + 1, lp, T.data());
            return cache.emplace(lp, std::move(T)).first->second;
        };
        std::vector<double> Mid(K2 * K2);
        for (int co = 0; co < 2; ++co)
            for (int ci = 0; ci < 2; ++ci) {
                const std::vector<double>& T = getT(2 * l + co - ci);
                for (int i = 0; i < k; ++i)
                    for (int j = 0; j < k; ++j) Mid[(co * k + i) * K2 + ci * k + j] = T[i * k + j];
            }
        const std::vector<double>& F = mra->basis.F;
        std::vector<double> tmp(K2 * K2, 0.0);
        for (int a = 0; a < K2; ++a)
            for (int b = 0; b < K2; ++b) {
                double s = 0.0;
                for (int c = 0; c < K2; ++c) s += F[a * K2 + c] * Mid[c * K2 + b];
                tmp[a * K2 + b] = s;
            }
        for (int a = 0; a < K2; ++a)
            for (int b = 0; b < K2; ++b) {
                double s = 0.0;
                for (int c = 0; c < K2; ++c) s += tmp[a * K2 + c] * F[b * K2 + c];
                NS[a * K2 + b] = s;
            }
    }

    // Build (once) the bands of all terms at a depth.  A term is kept at depth >= 1 only if its
    // largest possible block bound reaches cut(d) = 1e-6 eps B0 4^{-d}; its band extends while
    // beta * ||NS(l)|| * S^2 >= cut(d) (S = largest per-dimension block norm).
    std::vector<Band>& get_bands(int depth) {
        {
            std::lock_guard<std::mutex> g(mtx);
            auto it = bands.find(depth);
            if (it != bands.end()) return it->second;
        }
        const int k = mra->k();
        const int K2 = 2 * k;
        const int n = mra->n0 + depth;
        long extent = 0;
        for (int d = 0; d < 3; ++d) extent = std::max<long>(extent, (long)mra->boxes[d] << depth);
        double cut = (depth == 0) ? 0.0 : 1e-6 * eps * B0 * std::pow(4.0, -depth);
        std::vector<Band> bs(terms.size());
#pragma omp parallel for schedule(dynamic, 1)
        for (size_t m = 0; m < terms.size(); ++m) {
            Band& b = bs[m];
            std::map<long, std::vector<double>> cache;
            std::vector<double> ns_l;
            std::vector<double> t2, x2;
            std::vector<std::vector<double>> mats;
            auto compute = [&](long l) {
                std::vector<double> NS(K2 * K2);
                ns_matrix(terms[m].alpha, n, l, cache, NS.data());
                double tt = 0.0, xx = 0.0;
                for (int a = 0; a < K2; ++a)
                    for (int c = 0; c < K2; ++c) {
                        double v = NS[a * K2 + c] * NS[a * K2 + c];
                        if (a < k && c < k) tt += v; else xx += v;
                    }
                mats.push_back(std::move(NS));
                t2.push_back(tt);
                x2.push_back(xx);
            };
            compute(0);
            compute(1);
            const double beta = terms[m].beta;
            double S2 = std::max(t2[0] + x2[0], t2[1] + x2[1]);
            if (depth > 0) {
                double xmax = std::sqrt(std::max(x2[0], x2[1]));
                if (beta * 10.0 * xmax * S2 < cut) { b.active = false; continue; }
            }
            long L = 1;
            while (L + 1 < extent) {
                double last = std::sqrt(t2[L] + x2[L]);
                if (depth > 0 && beta * last * S2 < cut) break;
                if (depth == 0 && last <= 1e-300) break;
                if (depth == 0 && last < 1e-17 * std::sqrt(S2)) break;
                compute(L + 1);
                S2 = std::max(S2, t2[L + 1] + x2[L + 1]);
                ++L;
            }
            // trim the tail below the cut
            while (L > 0 && depth > 0 && beta * std::sqrt(t2[L] + x2[L]) * S2 < cut) --L;
            if (L >= extent) L = extent - 1;
            b.active = true;
            b.L = (int)L;
            b.ns.assign((size_t)(2 * L + 1) * K2 * K2, 0.0);
            b.t2.assign(2 * L + 1, 0.0);
            b.x2.assign(2 * L + 1, 0.0);
            for (long l = -L; l <= L; ++l) {
                long al = l < 0 ? -l : l;
                double* dst = &b.ns[(size_t)(l + L) * K2 * K2];
                const std::vector<double>& src = mats[al];
                for (int a = 0; a < K2; ++a)
                    for (int c = 0; c < K2; ++c)
                        dst[a * K2 + c] = (l >= 0) ? src[a * K2 + c] : src[c * K2 + a];  // NS(-l) = NS(l)^T
                b.t2[l + L] = t2[al];
                b.x2[l + L] = x2[al];
            }
        }
        std::lock_guard<std::mutex> g(mtx);
        return bands.emplace(depth, std::move(bs)).first->second;
    }

    static double bound3(double beta, const double* t, const double* x, bool root) {
        if (root) return beta * std::sqrt((t[0] + x[0]) * (t[1] + x[1]) * (t[2] + x[2]));
        double v = x[0] * (t[1] + x[1]) * (t[2] + x[2]) + t[0] * x[1] * (t[2] + x[2]) + t[0] * t[1] * x[2];
        return beta * std::sqrt(v);
    }

    // Offsets of a depth with their surviving terms, sorted by bound (descending).
    std::vector<DeltaEntry>& get_deltas(int depth) {
        {
            std::lock_guard<std::mutex> g(mtx);
            auto it = deltas.find(depth);
            if (it != deltas.end()) return it->second;
        }
        std::vector<Band>& bs = get_bands(depth);
        const bool root = depth == 0;
        double cut = root ? 0.0 : 1e-6 * eps * B0 * std::pow(4.0, -depth);
        std::map<std::tuple<int, int, int>, std::vector<std::pair<double, int>>> acc;
        for (size_t m = 0; m < bs.size(); ++m) {
            const Band& b = bs[m];
            if (!b.active) continue;
            const double beta = terms[m].beta;
            double S2 = 0.0;
            for (int i = 0; i < 2 * b.L + 1; ++i) S2 = std::max(S2, b.t2[i] + b.x2[i]);
            for (int dx = -b.L; dx <= b.L; ++dx) {
                double ax = b.t2[dx + b.L] + b.x2[dx + b.L];
                if (!root && beta * std::sqrt(ax) * S2 < cut) continue;
                for (int dy = -b.L; dy <= b.L; ++dy) {
                    double ay = b.t2[dy + b.L] + b.x2[dy + b.L];
                    if (!root && beta * std::sqrt(ax * ay * S2) < cut) continue;
                    for (int dz = -b.L; dz <= b.L; ++dz) {
                        double t[3] = {b.t2[dx + b.L], b.t2[dy + b.L], b.t2[dz + b.L]};
                        double x[3] = {b.x2[dx + b.L], b.x2[dy + b.L], b.x2[dz + b.L]};
                        double bd = bound3(beta, t, x, root);
                        if (bd <= 0.0 || bd < cut) continue;
                        acc[std::make_tuple(dx, dy, dz)].push_back({bd, (int)m});
                    }
                }
            }
        }
        std::vector<DeltaEntry> out;
        out.reserve(acc.size());
        for (auto& kv : acc) {
            DeltaEntry e;
            e.d[0] = std::get<0>(kv.first);
            e.d[1] = std::get<1>(kv.first);
            e.d[2] = std::get<2>(kv.first);
            e.terms = std::move(kv.second);
            std::stable_sort(e.terms.begin(), e.terms.end(),
                             [](const std::pair<double, int>& a, const std::pair<double, int>& b) {
                                 return a.first > b.first || (a.first == b.first && a.second < b.second);
                             });
            e.maxb = e.terms.front().first;
            out.push_back(std::move(e));
        }
        std::stable_sort(out.begin(), out.end(),
                         [](const DeltaEntry& a, const DeltaEntry& b) { return a.maxb > b.maxb; });
        std::lock_guard<std::mutex> g(mtx);
        return deltas.emplace(depth, std::move(out)).first->second;
    }
};

// Screening factor: a (output, input, term) contribution is skipped when its bound is below
// kScreen times the split threshold of the output depth.
const double kScreen = 0.1;

// ---------------------------------------------------------------------------------------------
// Adaptive NS-form apply
// ---------------------------------------------------------------------------------------------

struct ApplyStats {
    long long triples = 0;       // contracted (output node, input node, term) triples
    long long triples_gen = 0;   // of which with a generated (scaling-only) input node
    int passes = 0;
    double g0 = 0.0;
    long long lines_yz = 0;      // distinct (output node, term, dy, dz) among the triples
    long long lines_z = 0;       // distinct (output node, term, dz)
};

// s-only block of the generated input node (depth, t) below the leaf `leaf` (k^3 values)
void generate_node(const Tree& inp, int leaf, int depth, const int64_t t[3], double* s) {
    const MRA& mra = *inp.mra;
    const int k = mra.k();
    const int K2 = 2 * k;
    const Node& L = inp.nodes[leaf];
    std::vector<double> rec((size_t)K2 * K2 * K2);
    transform3(mra.basis.F, k, true, L.c.data(), rec.data());
    int dl = depth - L.depth;  // >= 1
    // child of the leaf on the path
    int64_t tc[3];
    for (int d = 0; d < 3; ++d) tc[d] = t[d] >> (dl - 1);
    int cc[3];
    for (int d = 0; d < 3; ++d) cc[d] = (int)(tc[d] - 2 * L.t[d]);
    std::vector<double> cur((size_t)k * k * k), nxt((size_t)k * k * k), tmp((size_t)k * k * k);
    for (int z = 0; z < k; ++z)
        for (int y = 0; y < k; ++y)
            for (int x = 0; x < k; ++x)
                cur[x + k * (y + k * z)] = rec[(cc[0] * k + x) + K2 * ((cc[1] * k + y) + K2 * (cc[2] * k + z))];
    // descend with zero wavelets: child c scaling = H_c^T s per dimension
    for (int lev = dl - 2; lev >= 0; --lev) {
        int c[3];
        for (int d = 0; d < 3; ++d) c[d] = (int)((t[d] >> lev) & 1);
        std::vector<double> M[3];
        for (int d = 0; d < 3; ++d) {
            M[d].assign(k * k, 0.0);
            for (int i = 0; i < k; ++i)
                for (int j = 0; j < k; ++j) M[d][i * k + j] = mra.basis.F[j * K2 + c[d] * k + i];
        }
        mode_product(M[0].data(), k, k, k, 0, cur.data(), k, k, k, tmp.data());
        mode_product(M[1].data(), k, k, k, 1, tmp.data(), k, k, k, nxt.data());
        mode_product(M[2].data(), k, k, k, 2, nxt.data(), k, k, k, cur.data());
    }
    std::memcpy(s, cur.data(), sizeof(double) * k * k * k);
}

void apply(double prec, Tree& out, Operator& op, const Tree& inp, ApplyStats* stats, bool line_order = false) {
    const MRA& mra = *inp.mra;
    const int k = mra.k();
    const int K2 = 2 * k;
    const size_t BS = mra.bsize();
    const size_t SS = (size_t)k * k * k;
    out.mra = inp.mra;
    out.make_roots();
    double fnorm = std::sqrt(inp.square_norm());
    double nu_max = 0.0;
    std::vector<double> inorm(inp.nodes.size());
    for (size_t i = 0; i < inp.nodes.size(); ++i) {
        inorm[i] = std::sqrt(sq_norm(inp.nodes[i].c.data(), BS));
        nu_max = std::max(nu_max, inorm[i]);
    }
    std::vector<int> work(out.nodes.size());
    for (size_t i = 0; i < work.size(); ++i) work[i] = (int)i;
    double g0 = 0.0;
    long long n_trip = 0, n_gen = 0, n_lyz = 0, n_lz = 0;
    int passes = 0;
    for (int depth = 0; !work.empty(); ++depth) {
        ++passes;
        const bool root = depth == 0;
        std::vector<DeltaEntry>& dl = op.get_deltas(depth);
        std::vector<Band>& bs = op.get_bands(depth);
        double theta;
        if (root) {
            double nu0 = dl.empty() ? 0.0 : dl.front().maxb;
            theta = kScreen * prec * fnorm * nu0;
        } else {
            theta = kScreen * split_threshold(prec, g0, depth);
        }
        // Phase A: candidate inputs per output node; collect generated nodes
        struct Cand { int delta; int src; };  // src >= 0 real node, src < 0 -> gen id -(src+1)
        std::vector<std::vector<Cand>> cands(work.size());
        std::vector<std::vector<std::pair<Key, std::pair<int, std::array<int64_t, 3>>>>> genreq(work.size());
        long long ext[3];
        for (int d = 0; d < 3; ++d) ext[d] = (long long)mra.boxes[d] << depth;
#pragma omp parallel for schedule(dynamic, 4)
        for (size_t q = 0; q < work.size(); ++q) {
            const Node& o = out.nodes[work[q]];
            for (size_t e = 0; e < dl.size(); ++e) {
                if (!(nu_max > 0.0) || dl[e].maxb * nu_max < theta) break;
                int64_t ti[3];
                bool inside = true;
                for (int d = 0; d < 3; ++d) {
                    ti[d] = o.t[d] - dl[e].d[d];
                    if (ti[d] < 0 || ti[d] >= ext[d]) inside = false;
                }
                if (!inside) continue;
                int idx = inp.find(depth, ti);
                if (idx >= 0) {
                    if (!(inorm[idx] > 0.0) || dl[e].maxb * inorm[idx] < theta) continue;
                    cands[q].push_back({(int)e, idx});
                } else {
                    int leaf = -1;
                    for (int da = depth - 1; da >= 0 && leaf < 0; --da) {
                        int64_t ta[3] = {ti[0] >> (depth - da), ti[1] >> (depth - da), ti[2] >> (depth - da)};
                        leaf = inp.find(da, ta);
                    }
                    if (leaf < 0) continue;
                    if (!(inorm[leaf] > 0.0) || dl[e].maxb * inorm[leaf] < theta) continue;  // ||gen|| <= ||leaf||
                    cands[q].push_back({(int)e, -1});
                    genreq[q].push_back({node_key(depth, ti), {leaf, {ti[0], ti[1], ti[2]}}});
                }
            }
        }
        auto keyless = [](const Key& x, const Key& y) { return x.a < y.a || (x.a == y.a && x.b < y.b); };
        std::map<Key, std::pair<int, std::array<int64_t, 3>>, decltype(keyless)> genmap(keyless);
        for (auto& v : genreq)
            for (auto& g : v) genmap.emplace(g.first, g.second);
        std::vector<Key> genkeys;
        for (auto& kv : genmap) genkeys.push_back(kv.first);
        std::unordered_map<Key, int, KeyHash> genid;
        for (size_t i = 0; i < genkeys.size(); ++i) genid[genkeys[i]] = (int)i;
        std::vector<double> gblk(genkeys.size() * SS);
        std::vector<double> gnorm(genkeys.size());
#pragma omp parallel for schedule(dynamic, 8)
        for (size_t i = 0; i < genkeys.size(); ++i) {
            auto& g = genmap[genkeys[i]];
            generate_node(inp, g.first, depth, g.second.data(), &gblk[i * SS]);
            gnorm[i] = std::sqrt(sq_norm(&gblk[i * SS], SS));
        }
        // fill gen ids
        for (size_t q = 0; q < work.size(); ++q) {
            size_t gi = 0;
            for (Cand& c : cands[q])
                if (c.src < 0) c.src = -(genid[genreq[q][gi++].first] + 1);
        }
        // Phase B: contractions
        std::vector<long long> trip(work.size(), 0), tripg(work.size(), 0), lyz(work.size(), 0), lz(work.size(), 0);
#pragma omp parallel for schedule(dynamic, 1)
        for (size_t q = 0; q < work.size(); ++q) {
            Node& o = out.nodes[work[q]];
            std::vector<double> acc(BS, 0.0), t1(BS), t2(BS), t3(BS);
            std::vector<double> s_in(SS), u1(SS), u2(SS), u3(SS);
            std::vector<std::array<int, 3>> seen_yz, seen_z;
            if (line_order) {
                // The same triples summed in line order (the order of the GPU's line-ordered
                // contraction): sorted by (term, dz, dy), a line's x products are summed before its y
                // product and a plane's y products before its z product.  Linear algebra makes this
                // the same sum in another order.
                struct Tri { int m, dz, dy, c; };
                std::vector<Tri> tri;
                for (int ci = 0; ci < (int)cands[q].size(); ++ci) {
                    const Cand& c = cands[q][ci];
                    const DeltaEntry& de = dl[c.delta];
                    const double nu = c.src < 0 ? gnorm[-c.src - 1] : inorm[c.src];
                    if (!(nu > 0.0) || de.maxb * nu < theta) continue;
                    for (const auto& tb : de.terms) {
                        if (tb.first * nu < theta) break;
                        tri.push_back({tb.second, de.d[2], de.d[1], ci});
                    }
                }
                std::stable_sort(tri.begin(), tri.end(), [](const Tri& a, const Tri& b) {
                    return a.m != b.m ? a.m < b.m : a.dz != b.dz ? a.dz < b.dz : a.dy < b.dy;
                });
                std::vector<double> full(BS), line(BS), plane(BS), tmp(BS), sline(SS), splane(SS), stmp(SS);
                size_t t = 0;
                while (t < tri.size()) {
                    const int m = tri[t].m, dz = tri[t].dz;
                    const Band& b = bs[m];
                    const double beta = op.terms[m].beta;
                    std::fill(plane.begin(), plane.end(), 0.0);
                    std::fill(splane.begin(), splane.end(), 0.0);
                    while (t < tri.size() && tri[t].m == m && tri[t].dz == dz) {
                        const int dy = tri[t].dy;
                        std::fill(line.begin(), line.end(), 0.0);
                        std::fill(sline.begin(), sline.end(), 0.0);
                        while (t < tri.size() && tri[t].m == m && tri[t].dz == dz && tri[t].dy == dy) {
                            const Cand& c = cands[q][tri[t].c];
                            const DeltaEntry& de = dl[c.delta];
                            const bool gen = c.src < 0;
                            if (gen) {  // the scaling-only block, zero elsewhere
                                const double* g = &gblk[(size_t)(-c.src - 1) * SS];
                                std::fill(full.begin(), full.end(), 0.0);
                                for (int z = 0; z < k; ++z)
                                    for (int y = 0; y < k; ++y)
                                        for (int x = 0; x < k; ++x) full[x + K2 * (y + K2 * z)] = g[x + k * (y + k * z)];
                            } else {
                                std::copy(inp.nodes[c.src].c.begin(), inp.nodes[c.src].c.end(), full.begin());
                            }
                            const double* Mx = &b.ns[(size_t)(de.d[0] + b.L) * K2 * K2];
                            mode_product(Mx, K2, K2, K2, 0, full.data(), K2, K2, K2, tmp.data());
                            for (size_t i = 0; i < BS; ++i) line[i] += tmp[i];
                            if (!root) {
                                for (int z = 0; z < k; ++z)
                                    for (int y = 0; y < k; ++y)
                                        for (int x = 0; x < k; ++x) s_in[x + k * (y + k * z)] = full[x + K2 * (y + K2 * z)];
                                mode_product(Mx, K2, k, k, 0, s_in.data(), k, k, k, stmp.data());
                                for (size_t i = 0; i < SS; ++i) sline[i] += stmp[i];
                            }
                            ++trip[q];
                            if (gen) ++tripg[q];
                            seen_yz.push_back({m, dy, dz});
                            seen_z.push_back({m, 0, dz});
                            ++t;
                        }
                        const double* My = &b.ns[(size_t)(dy + b.L) * K2 * K2];
                        mode_product(My, K2, K2, K2, 1, line.data(), K2, K2, K2, tmp.data());
                        for (size_t i = 0; i < BS; ++i) plane[i] += tmp[i];
                        if (!root) {
                            mode_product(My, K2, k, k, 1, sline.data(), k, k, k, stmp.data());
                            for (size_t i = 0; i < SS; ++i) splane[i] += stmp[i];
                        }
                    }
                    const double* Mz = &b.ns[(size_t)(dz + b.L) * K2 * K2];
                    mode_product(Mz, K2, K2, K2, 2, plane.data(), K2, K2, K2, tmp.data());
                    for (size_t i = 0; i < BS; ++i) acc[i] += beta * tmp[i];
                    if (!root) {  // remove the scaling->scaling block (it belongs to the coarser scale)
                        mode_product(Mz, K2, k, k, 2, splane.data(), k, k, k, u3.data());
                        for (int z = 0; z < k; ++z)
                            for (int y = 0; y < k; ++y)
                                for (int x = 0; x < k; ++x) acc[x + K2 * (y + K2 * z)] -= beta * u3[x + k * (y + k * z)];
                    }
                }
            } else
            for (const Cand& c : cands[q]) {
                const DeltaEntry& de = dl[c.delta];
                const bool gen = c.src < 0;
                const double* blk = gen ? &gblk[(size_t)(-c.src - 1) * SS] : inp.nodes[c.src].c.data();
                const double nu = gen ? gnorm[-c.src - 1] : inorm[c.src];
                if (!(nu > 0.0) || de.maxb * nu < theta) continue;
                if (!gen && !root) {
                    for (int z = 0; z < k; ++z)
                        for (int y = 0; y < k; ++y)
                            for (int x = 0; x < k; ++x) s_in[x + k * (y + k * z)] = blk[x + K2 * (y + K2 * z)];
                }
                for (const auto& tb : de.terms) {
                    if (tb.first * nu < theta) break;
                    const int m = tb.second;
                    const Band& b = bs[m];
                    const double beta = op.terms[m].beta;
                    const double* Mx = &b.ns[(size_t)(de.d[0] + b.L) * K2 * K2];
                    const double* My = &b.ns[(size_t)(de.d[1] + b.L) * K2 * K2];
                    const double* Mz = &b.ns[(size_t)(de.d[2] + b.L) * K2 * K2];
                    if (gen) {
                        mode_product(Mx, K2, K2, k, 0, blk, k, k, k, t1.data());
                        mode_product(My, K2, K2, k, 1, t1.data(), K2, k, k, t2.data());
                        mode_product(Mz, K2, K2, k, 2, t2.data(), K2, K2, k, t3.data());
                    } else {
                        mode_product(Mx, K2, K2, K2, 0, blk, K2, K2, K2, t1.data());
                        mode_product(My, K2, K2, K2, 1, t1.data(), K2, K2, K2, t2.data());
                        mode_product(Mz, K2, K2, K2, 2, t2.data(), K2, K2, K2, t3.data());
                    }
                    for (size_t i = 0; i < BS; ++i) acc[i] += beta * t3[i];
                    if (!root) {
                        // remove the scaling->scaling block (it belongs to the coarser scale)
                        const double* src = gen ? blk : s_in.data();
                        mode_product(Mx, K2, k, k, 0, src, k, k, k, u1.data());
                        mode_product(My, K2, k, k, 1, u1.data(), k, k, k, u2.data());
                        mode_product(Mz, K2, k, k, 2, u2.data(), k, k, k, u3.data());
                        for (int z = 0; z < k; ++z)
                            for (int y = 0; y < k; ++y)
                                for (int x = 0; x < k; ++x)
                                    acc[x + K2 * (y + K2 * z)] -= beta * u3[x + k * (y + k * z)];
                    }
                    ++trip[q];
                    if (gen) ++tripg[q];
                    seen_yz.push_back({m, de.d[1], de.d[2]});
                    seen_z.push_back({m, 0, de.d[2]});
                }
            }
            o.c = acc;
            std::sort(seen_yz.begin(), seen_yz.end());
            std::sort(seen_z.begin(), seen_z.end());
            lyz[q] = std::unique(seen_yz.begin(), seen_yz.end()) - seen_yz.begin();
            lz[q] = std::unique(seen_z.begin(), seen_z.end()) - seen_z.begin();
        }
        for (size_t q = 0; q < work.size(); ++q) {
            n_trip += trip[q];
            n_gen += tripg[q];
            n_lyz += lyz[q];
            n_lz += lz[q];
        }
        if (root) {
            double s = 0.0;
            for (int i : work) s += sq_norm(out.nodes[i].c.data(), BS);
            g0 = std::sqrt(s);
        }
        std::vector<int> next;
        if (prec > 0.0 && g0 > 0.0) {
            double thr = split_threshold(prec, g0, depth);
            for (int i : work) {
                if (out.nodes[i].depth >= mra.max_depth) continue;
                double w = std::sqrt(wavelet_sq_norm(out.nodes[i].c.data(), k));
                if (w > thr) {
                    out.split(i);
                    int c0 = out.nodes[i].child0;
                    for (int c = 0; c < 8; ++c) next.push_back(c0 + c);
                }
            }
        }
        work.swap(next);
    }
    // Sum-up: top-down accumulation of the scaling parts, then bottom-up compression.
    std::vector<int> ord = out.level_order();
    std::vector<double> rec(BS);
    for (int i : ord) {
        Node& nd = out.nodes[i];
        if (nd.child0 < 0) continue;
        transform3(mra.basis.F, k, true, nd.c.data(), rec.data());
        for (int c = 0; c < 8; ++c) {
            Node& ch = out.nodes[nd.child0 + c];
            int cx = c & 1, cy = (c >> 1) & 1, cz = (c >> 2) & 1;
            for (int z = 0; z < k; ++z)
                for (int y = 0; y < k; ++y)
                    for (int x = 0; x < k; ++x)
                        ch.c[x + K2 * (y + K2 * z)] += rec[(cx * k + x) + K2 * ((cy * k + y) + K2 * (cz * k + z))];
        }
    }
    compress_bottom_up(out);
    if (stats) {
        stats->triples = n_trip;
        stats->triples_gen = n_gen;
        stats->passes = passes;
        stats->g0 = g0;
        stats->lines_yz = n_lyz;
        stats->lines_z = n_lz;
    }
}

// <a|b> of two compressed trees on the same world
double dot(const Tree& a, const Tree& b) {
    const int k = a.mra->k();
    const int K2 = 2 * k;
    double s = 0.0;
    for (const Node& na : a.nodes) {
        int j = b.find(na.depth, na.t);
        if (j < 0) continue;
        const Node& nb = b.nodes[j];
        for (int z = 0; z < K2; ++z)
            for (int y = 0; y < K2; ++y)
                for (int x = 0; x < K2; ++x) {
                    bool scal = x < k && y < k && z < k;
                    if (scal && na.depth > 0) continue;
                    size_t i = x + K2 * (y + (size_t)K2 * z);
                    s += na.c[i] * nb.c[i];
                }
    }
    return s;
}

// point value from the leaf containing r
double evalf(const Tree& tr, const double* r) {
    const MRA& mra = *tr.mra;
    const int k = mra.k();
    const int K2 = 2 * k;
    double root_edge = std::ldexp(1.0, -mra.n0);
    int64_t t[3];
    for (int d = 0; d < 3; ++d) {
        double u = (r[d] - mra.corner[d] * root_edge) / root_edge;
        t[d] = (int64_t)std::floor(u);
        if (t[d] < 0 || t[d] >= mra.boxes[d]) return 0.0;
    }
    int idx = tr.find(0, t);
    while (idx >= 0 && tr.nodes[idx].child0 >= 0) {
        const Node& nd = tr.nodes[idx];
        double edge = std::ldexp(root_edge, -nd.depth);
        int c = 0;
        for (int d = 0; d < 3; ++d) {
            double lo = mra.corner[d] * root_edge + nd.t[d] * edge;
            if (r[d] - lo >= 0.5 * edge) c |= (1 << d);
        }
        idx = nd.child0 + c;
    }
    if (idx < 0) return 0.0;
    const Node& nd = tr.nodes[idx];
    std::vector<double> rec(mra.bsize());
    transform3(mra.basis.F, k, true, nd.c.data(), rec.data());
    int n1 = mra.n0 + nd.depth + 1;
    double edge = std::ldexp(1.0, -n1);
    int cc[3];
    double u[3];
    for (int d = 0; d < 3; ++d) {
        double lo = mra.corner[d] * root_edge + 2 * nd.t[d] * edge;
        double v = (r[d] - lo) / edge;
        cc[d] = v >= 1.0 ? 1 : 0;
        u[d] = v - cc[d];
    }
    std::vector<double> px(k), py(k), pz(k);
    mra.basis.phi_all(u[0], px.data());
    mra.basis.phi_all(u[1], py.data());
    mra.basis.phi_all(u[2], pz.data());
    double s = 0.0;
    for (int z = 0; z < k; ++z)
        for (int y = 0; y < k; ++y)
            for (int x = 0; x < k; ++x)
                s += rec[(cc[0] * k + x) + K2 * ((cc[1] * k + y) + K2 * (cc[2] * k + z))] * px[x] * py[y] * pz[z];
    return s * std::pow(2.0, 1.5 * n1);
}

// ---------------------------------------------------------------------------------------------
// Pointwise product of two functions (multiwavelet multiplication)
// ---------------------------------------------------------------------------------------------
// Contract: mrcpp::multiply(prec, out, c, a, b[, maxIter]) as called at
// src/qmfunctions/qmfunction_utils.cpp:209-217 (union grid: build_grid(out, a), build_grid(out, b),
// then multiply with maxIter = 0; adaptive: multiply on the output's current grid, refined until
// converged) and src/qmoperators/two_electron/ExchangePotential.cpp:131,253,312.
// Method (restated from the MW literature, not from MRCPP): for an output node at scale n both
// factors are taken at scale n+1 on the node's 8 children -- the reconstructed node block, or, where
// a factor's tree is coarser, the block generated below its deepest existing ancestor (zero
// wavelets) -- evaluated at the children's k^3 Gauss-Legendre points, multiplied, projected back
// with the quadrature of the adaptive projection and compressed into the node block.  Refinement
// uses the projection's wavelet criterion with the norm of the current product.

// compressed block of `tr` at (depth, t): the node's own block, or the scaling-only block generated
// below the deepest existing ancestor (a leaf)
void block_at(const Tree& tr, int depth, const int64_t t[3], double* out) {
    const MRA& mra = *tr.mra;
    const int k = mra.k(), K2 = 2 * k;
    const size_t BS = mra.bsize();
    const int idx = tr.find(depth, t);
    if (idx >= 0) {
        std::memcpy(out, tr.nodes[idx].c.data(), sizeof(double) * BS);
        return;
    }
    int leaf = -1;
    for (int da = depth - 1; da >= 0 && leaf < 0; --da) {
        int64_t ta[3] = {t[0] >> (depth - da), t[1] >> (depth - da), t[2] >> (depth - da)};
        leaf = tr.find(da, ta);
    }
    std::fill(out, out + BS, 0.0);
    if (leaf < 0) return;
    std::vector<double> s((size_t)k * k * k);
    generate_node(tr, leaf, depth, t, s.data());
    for (int z = 0; z < k; ++z)
        for (int y = 0; y < k; ++y)
            for (int x = 0; x < k; ++x) out[x + K2 * (y + K2 * z)] = s[x + k * (y + k * z)];
}

// block of the product c a b at output node (depth, t)
void multiply_node(const MRA& mra, double c, const Tree& a, const Tree& b, int depth, const int64_t t[3],
                   double* out) {
    const int k = mra.k(), K2 = 2 * k;
    const size_t BS = mra.bsize();
    const Basis& B = mra.basis;
    // EE = blockdiag(E, E), E[q][j] = phi_j(x_q);  WW = blockdiag(W, W), W[j][q] = w_q phi_j(x_q)
    std::vector<double> EE((size_t)K2 * K2, 0.0), WW((size_t)K2 * K2, 0.0);
    for (int h = 0; h < 2; ++h)
        for (int q = 0; q < k; ++q)
            for (int j = 0; j < k; ++j) {
                const double pj = B.phi(j, B.qx[q]);
                EE[(h * k + q) * K2 + h * k + j] = pj;
                WW[(h * k + j) * K2 + h * k + q] = B.qw[q] * pj;
            }
    std::vector<double> ba(BS), bb(BS), ra(BS), rb(BS), va(BS), vb(BS);
    block_at(a, depth, t, ba.data());
    block_at(b, depth, t, bb.data());
    transform3(B.F, k, true, ba.data(), ra.data());
    transform3(B.F, k, true, bb.data(), rb.data());
    transform3(EE, k, false, ra.data(), va.data());
    transform3(EE, k, false, rb.data(), vb.data());
    for (size_t i = 0; i < BS; ++i) va[i] *= vb[i];
    transform3(WW, k, false, va.data(), ra.data());
    const double fac = c * std::pow(2.0, 1.5 * (mra.n0 + depth + 1));
    for (size_t i = 0; i < BS; ++i) ra[i] *= fac;
    transform3(B.F, k, false, ra.data(), out);
}

// out = c a b.  `out` keeps its current grid (roots if empty); every leaf is computed, then leaves
// whose wavelet norm exceeds prec ||out|| 2^{-depth/2} are split and their children computed, at
// most max_iter times (max_iter < 0: until no split; prec <= 0: no refinement).
void multiply(double prec, Tree& out, double c, const Tree& a, const Tree& b, int max_iter) {
    const MRA& mra = *a.mra;
    out.mra = a.mra;
    if (out.nodes.empty()) out.make_roots();
    std::vector<int> work;
    for (int i : out.level_order())
        if (out.nodes[i].child0 < 0) work.push_back(i);
    for (int iter = 0; !work.empty(); ++iter) {
#pragma omp parallel for schedule(dynamic, 1)
        for (size_t q = 0; q < work.size(); ++q) {
            Node& nd = out.nodes[work[q]];
            multiply_node(mra, c, a, b, nd.depth, nd.t, nd.c.data());
        }
        if (prec <= 0.0 || (max_iter >= 0 && iter >= max_iter)) break;
        const double ref = std::sqrt(out.square_norm());
        std::vector<int> next;
        for (int i : work) {
            const Node& nd = out.nodes[i];
            if (nd.depth >= mra.max_depth) continue;
            const double w = std::sqrt(wavelet_sq_norm(nd.c.data(), mra.k()));
            if (w > split_threshold(prec, ref, nd.depth)) {
                out.split(i);
                const int c0 = out.nodes[i].child0;
                for (int ch = 0; ch < 8; ++ch) next.push_back(c0 + ch);
            }
        }
        work.swap(next);
    }
    compress_bottom_up(out);
}

// ---------------------------------------------------------------------------------------------
// First-derivative operator (Alpert, Beylkin, Gines & Vozovoi 2002), contract of
// mrcpp::ABGVOperator<3>(MRA, a, b) + mrcpp::apply(out, D, inp, dir) (reference src/SCFDriver.cpp:282,
// src/qmoperators/one_electron/NablaOperator.cpp:35).  Flux: at the right interface of a cell
// f = (1-a) f_left + a f_right, at the left interface f = b f_left + (1-b) f_right; integrating
// phi_i f' by parts on the cell gives the unit-scale blocks for output cell l, input cell l - d:
//   T(0) = (1-a) phi(1) phi(1)^T - (1-b) phi(0) phi(0)^T - <phi', phi>,
//   T(-1) = a phi(1) phi(0)^T,  T(+1) = -b phi(0) phi(1)^T,  scaled by 2^n at scale n.
// The apply is the non-standard form on the input's grid: for each node, the derivative's NS matrix
// of the offset along dir (identity along the other directions) on the input blocks of the same
// scale (own or generated), the s->s block removed below the root, then sum-up and compression.
// ---------------------------------------------------------------------------------------------
void derivative_unit_blocks(const Basis& B, double a, double b, std::vector<double> T[3]) {
    const int k = B.k;
    std::vector<double> p0(k), p1(k);
    for (int j = 0; j < k; ++j) {
        p0[j] = B.phi(j, 0.0);
        p1[j] = B.phi(j, 1.0);
    }
    for (int d = 0; d < 3; ++d) T[d].assign((size_t)k * k, 0.0);
    for (int i = 0; i < k; ++i)
        for (int j = 0; j < k; ++j) {
            double I = 0.0;
            for (int q = 0; q < k; ++q) I += B.qw[q] * B.dphi(i, B.qx[q]) * B.phi(j, B.qx[q]);
            T[1][i * k + j] = (1.0 - a) * p1[i] * p1[j] - (1.0 - b) * p0[i] * p0[j] - I;
            T[0][i * k + j] = a * p1[i] * p0[j];
            T[2][i * k + j] = -b * p0[i] * p1[j];
        }
}

// NS matrix of the derivative at depth, offset l: F [[T(2l) T(2l-1)]; [T(2l+1) T(2l)]] F^T with the
// children-scale blocks 2^{n+1} T_unit
std::vector<double> derivative_ns(const MRA& mra, const std::vector<double> T[3], int depth, int l) {
    const int k = mra.k(), K2 = 2 * k;
    const double fac = std::ldexp(1.0, mra.n0 + depth + 1);
    std::vector<double> C((size_t)K2 * K2, 0.0), NS((size_t)K2 * K2, 0.0), tmp((size_t)K2 * K2, 0.0);
    for (int co = 0; co < 2; ++co)
        for (int ci = 0; ci < 2; ++ci) {
            const int d = 2 * l + co - ci;
            if (d < -1 || d > 1) continue;
            for (int i = 0; i < k; ++i)
                for (int j = 0; j < k; ++j) C[(size_t)(co * k + i) * K2 + ci * k + j] = fac * T[d + 1][i * k + j];
        }
    const std::vector<double>& F = mra.basis.F;
    for (int a = 0; a < K2; ++a)
        for (int c = 0; c < K2; ++c)
            for (int b = 0; b < K2; ++b) tmp[(size_t)a * K2 + c] += F[(size_t)a * K2 + b] * C[(size_t)b * K2 + c];
    for (int a = 0; a < K2; ++a)
        for (int c = 0; c < K2; ++c)
            for (int b = 0; b < K2; ++b) NS[(size_t)a * K2 + c] += tmp[(size_t)a * K2 + b] * F[(size_t)c * K2 + b];
    return NS;
}

void derivative_apply(Tree& out, const Tree& inp, double a, double b, int dir) {
    const MRA& mra = *inp.mra;
    const int k = mra.k(), K2 = 2 * k;
    const size_t BS = mra.bsize(), SS = (size_t)k * k * k;
    std::vector<double> T[3];
    derivative_unit_blocks(mra.basis, a, b, T);
    // the input's grid
    out.mra = inp.mra;
    out.clear();
    for (const Node& nd : inp.nodes) {
        Node c;
        c.depth = nd.depth;
        for (int d = 0; d < 3; ++d) c.t[d] = nd.t[d];
        c.parent = nd.parent;
        c.child0 = nd.child0;
        c.c.assign(BS, 0.0);
        out.nodes.push_back(std::move(c));
        out.index[node_key(nd.depth, nd.t)] = (int)out.nodes.size() - 1;
    }
    std::map<std::pair<int, int>, std::vector<double>> ns;  // (depth, l) -> NS matrix
    int maxd = out.max_depth_present();
    for (int d = 0; d <= maxd; ++d)
        for (int l = -1; l <= 1; ++l) ns[{d, l}] = derivative_ns(mra, T, d, l);
#pragma omp parallel for schedule(dynamic, 4)
    for (size_t q = 0; q < out.nodes.size(); ++q) {
        Node& o = out.nodes[q];
        std::vector<double> blk(BS), t1(BS), sin(SS), u1(SS);
        const long long ext = (long long)mra.boxes[dir] << o.depth;
        for (int l = -1; l <= 1; ++l) {
            int64_t ti[3] = {o.t[0], o.t[1], o.t[2]};
            ti[dir] -= l;
            if (ti[dir] < 0 || ti[dir] >= ext) continue;
            block_at(inp, o.depth, ti, blk.data());
            const std::vector<double>& M = ns[{o.depth, l}];
            mode_product(M.data(), K2, K2, K2, dir, blk.data(), K2, K2, K2, t1.data());
            for (size_t i = 0; i < BS; ++i) o.c[i] += t1[i];
            if (o.depth > 0) {  // remove the scaling->scaling block
                for (int z = 0; z < k; ++z)
                    for (int y = 0; y < k; ++y)
                        for (int x = 0; x < k; ++x) sin[x + k * (y + k * z)] = blk[x + K2 * (y + K2 * z)];
                mode_product(M.data(), K2, k, k, dir, sin.data(), k, k, k, u1.data());
                for (int z = 0; z < k; ++z)
                    for (int y = 0; y < k; ++y)
                        for (int x = 0; x < k; ++x) o.c[x + K2 * (y + K2 * z)] -= u1[x + k * (y + k * z)];
            }
        }
    }
    // sum-up top-down, then compression
    std::vector<double> rec(BS);
    for (int i : out.level_order()) {
        Node& nd = out.nodes[i];
        if (nd.child0 < 0) continue;
        transform3(mra.basis.F, k, true, nd.c.data(), rec.data());
        for (int c = 0; c < 8; ++c) {
            Node& ch = out.nodes[nd.child0 + c];
            int cx = c & 1, cy = (c >> 1) & 1, cz = (c >> 2) & 1;
            for (int z = 0; z < k; ++z)
                for (int y = 0; y < k; ++y)
                    for (int x = 0; x < k; ++x)
                        ch.c[x + K2 * (y + K2 * z)] += rec[(cx * k + x) + K2 * ((cy * k + y) + K2 * (cz * k + z))];
        }
    }
    compress_bottom_up(out);
}

// out = sum_i c_i f_i (mrcpp::add(prec, out, vec[, maxIter]) contract: reference
// src/qmfunctions/qmfunction_utils.cpp:170-177, src/qmfunctions/density_utils.cpp:87,
// src/mrdft/XCFunctional.cpp:713, src/scf_solver/KAIN.cpp:180,192).  Compressed blocks are linear in
// the function, so a node's block is the combination of the inputs' blocks at that node (their own, or
// generated below their deepest ancestor); grid and refinement as in multiply().
void add(double prec, Tree& out, const std::vector<double>& c, const std::vector<const Tree*>& f, int max_iter) {
    const MRA& mra = *f[0]->mra;
    const size_t BS = mra.bsize();
    out.mra = f[0]->mra;
    if (out.nodes.empty()) out.make_roots();
    std::vector<int> work;
    for (int i : out.level_order())
        if (out.nodes[i].child0 < 0) work.push_back(i);
    for (int iter = 0; !work.empty(); ++iter) {
#pragma omp parallel for schedule(dynamic, 4)
        for (size_t q = 0; q < work.size(); ++q) {
            Node& nd = out.nodes[work[q]];
            std::vector<double> blk(BS);
            std::fill(nd.c.begin(), nd.c.end(), 0.0);
            for (size_t i = 0; i < f.size(); ++i) {
                block_at(*f[i], nd.depth, nd.t, blk.data());
                for (size_t e = 0; e < BS; ++e) nd.c[e] += c[i] * blk[e];
            }
        }
        if (prec <= 0.0 || (max_iter >= 0 && iter >= max_iter)) break;
        const double ref = std::sqrt(out.square_norm());
        std::vector<int> next;
        for (int i : work) {
            const Node& nd = out.nodes[i];
            if (nd.depth >= mra.max_depth) continue;
            const double w = std::sqrt(wavelet_sq_norm(nd.c.data(), mra.k()));
            if (w > split_threshold(prec, ref, nd.depth)) {
                out.split(i);
                const int c0 = out.nodes[i].child0;
                for (int ch = 0; ch < 8; ++ch) next.push_back(c0 + ch);
            }
        }
        work.swap(next);
    }
    compress_bottom_up(out);
}

// extend the grid of `out` by the grid of `inp` (union; new nodes have zero blocks)
void build_grid(Tree& out, const Tree& inp) {
    out.mra = inp.mra;
    if (out.nodes.empty()) out.make_roots();
    for (int i : inp.level_order()) {
        const Node& nd = inp.nodes[i];
        if (nd.depth == 0 || out.find(nd.depth, nd.t) >= 0) continue;
        int64_t tp[3] = {nd.t[0] >> 1, nd.t[1] >> 1, nd.t[2] >> 1};
        const int p = out.find(nd.depth - 1, tp);
        if (p >= 0 && out.nodes[p].child0 < 0) out.split(p);
    }
}

Func make_func(int type, const double* p) {
    Func f;
    if (type == 1) {
        int ng = (int)p[0];
        for (int g = 0; g < ng; ++g) {
            const double* q = p + 1 + 8 * g;
            Func::G G;
            G.c = q[0];
            G.a = q[1];
            G.R[0] = q[2]; G.R[1] = q[3]; G.R[2] = q[4];
            G.p[0] = (int)q[5]; G.p[1] = (int)q[6]; G.p[2] = (int)q[7];
            f.gs.push_back(G);
        }
    } else if (type == 2) {
        int nt = (int)p[0];
        for (int i = 0; i < nt; ++i) {
            const double* q = p + 1 + 11 * i;
            Func::HP h;
            h.c = q[0];
            h.A.n = (int)q[1]; h.A.l = (int)q[2]; h.A.m = (int)q[3];
            h.B.n = (int)q[4]; h.B.l = (int)q[5]; h.B.m = (int)q[6];
            h.A.Z = h.B.Z = q[7];
            for (int d = 0; d < 3; ++d) h.A.o[d] = h.B.o[d] = q[8 + d];
            h.hasB = h.B.n > 0;
            h.A.init();
            if (h.hasB) h.B.init();
            f.hs.push_back(h);
        }
    }
    return f;
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// C API (ctypes)
// ---------------------------------------------------------------------------------------------
extern "C" {

void* oracle_mra_create(int min_scale, const int* corner, const int* boxes, int basis_type, int order,
                        int max_depth) {
    MRA* m = new MRA;
    m->n0 = min_scale;
    for (int d = 0; d < 3; ++d) {
        m->corner[d] = corner[d];
        m->boxes[d] = boxes[d];
    }
    m->max_depth = max_depth;
    m->basis.build(basis_type, order);
    return m;
}
void oracle_mra_destroy(void* m) { delete (MRA*)m; }
int oracle_mra_filter(void* m, double* F) {
    MRA* mra = (MRA*)m;
    std::memcpy(F, mra->basis.F.data(), sizeof(double) * mra->basis.F.size());
    return 2 * mra->k();
}

void* oracle_tree_create(void* m) {
    Tree* t = new Tree;
    t->mra = (MRA*)m;
    return t;
}
void oracle_tree_destroy(void* t) { delete (Tree*)t; }

int oracle_project(void* t, double prec, int type, const double* params) {
    Tree* tr = (Tree*)t;
    Func f = make_func(type, params);
    project(*tr, f, prec);
    return (int)tr->nodes.size();
}

int oracle_tree_nnodes(void* t) { return (int)((Tree*)t)->nodes.size(); }
double oracle_tree_square_norm(void* t) { return ((Tree*)t)->square_norm(); }
double oracle_dot(void* a, void* b) { return dot(*(Tree*)a, *(Tree*)b); }
double oracle_evalf(void* t, const double* r) { return evalf(*(Tree*)t, r); }

// Export in the tree's own node order: depth, translation (3), parent, child0, coefficients.
void oracle_tree_export(void* t, int* depth, long long* trans, int* parent, int* child0, double* coef) {
    Tree* tr = (Tree*)t;
    size_t BS = tr->mra->bsize();
    for (size_t i = 0; i < tr->nodes.size(); ++i) {
        const Node& n = tr->nodes[i];
        depth[i] = n.depth;
        for (int d = 0; d < 3; ++d) trans[3 * i + d] = n.t[d];
        parent[i] = n.parent;
        child0[i] = n.child0;
        if (coef) std::memcpy(coef + i * BS, n.c.data(), sizeof(double) * BS);
    }
}

// Import nodes (parents must precede children; children of a node consecutive, c = cx+2cy+4cz).
int oracle_tree_import(void* t, int n, const int* depth, const long long* trans, const int* parent,
                       const int* child0, const double* coef) {
    Tree* tr = (Tree*)t;
    tr->clear();
    size_t BS = tr->mra->bsize();
    for (int i = 0; i < n; ++i) {
        Node nd;
        nd.depth = depth[i];
        for (int d = 0; d < 3; ++d) nd.t[d] = trans[3 * i + d];
        nd.parent = parent[i];
        nd.child0 = child0[i];
        nd.c.assign(coef + (size_t)i * BS, coef + (size_t)(i + 1) * BS);
        tr->nodes.push_back(std::move(nd));
        tr->index[node_key(depth[i], tr->nodes.back().t)] = i;
    }
    return 0;
}

void* oracle_operator_create(void* m, double mu, double prec) {
    Operator* op = new Operator;
    op->init((MRA*)m, mu, prec);
    return op;
}
void oracle_operator_destroy(void* o) { delete (Operator*)o; }
int oracle_operator_nterms(void* o) { return (int)((Operator*)o)->terms.size(); }
void oracle_operator_terms(void* o, double* alpha, double* beta) {
    Operator* op = (Operator*)o;
    for (size_t m = 0; m < op->terms.size(); ++m) {
        alpha[m] = op->terms[m].alpha;
        beta[m] = op->terms[m].beta;
    }
}
// NS matrix of term m at depth, offset l (returns 0 if outside the stored band)
int oracle_operator_ns(void* o, int depth, int m, int l, double* NS) {
    Operator* op = (Operator*)o;
    std::vector<Band>& bs = op->get_bands(depth);
    const Band& b = bs[m];
    int K2 = 2 * op->mra->k();
    if (!b.active || l < -b.L || l > b.L) return 0;
    std::memcpy(NS, &b.ns[(size_t)(l + b.L) * K2 * K2], sizeof(double) * K2 * K2);
    return 1;
}
// raw scaling-function matrix T^n(l) (k x k) for exp(-alpha x^2), computed on demand
void oracle_scaling_matrix(void* o, double alpha, int n, int l, double* T) {
    ((Operator*)o)->scaling_matrix(alpha, n, l, T);
}

int oracle_apply_ordered(double prec, void* out, void* op, void* inp, long long* stats, int line_order);
int oracle_apply(double prec, void* out, void* op, void* inp, long long* stats) {
    return oracle_apply_ordered(prec, out, op, inp, stats, 0);
}
// line_order != 0: the per-node sums in the line order of the GPU contraction (same triples)
int oracle_apply_ordered(double prec, void* out, void* op, void* inp, long long* stats, int line_order) {
    ApplyStats st;
    apply(prec, *(Tree*)out, *(Operator*)op, *(Tree*)inp, &st, line_order != 0);
    if (stats) {
        stats[0] = st.triples;
        stats[1] = st.triples_gen;
        stats[2] = st.passes;
        stats[3] = st.lines_yz;
        stats[4] = st.lines_z;
    }
    return (int)((Tree*)out)->nodes.size();
}

// out = c a b (mrcpp::multiply contract); returns the number of output nodes
int oracle_multiply(double prec, void* out, double c, void* a, void* b, int max_iter) {
    multiply(prec, *(Tree*)out, c, *(Tree*)a, *(Tree*)b, max_iter);
    return (int)((Tree*)out)->nodes.size();
}
// out = sum_i c[i] f[i] (mrcpp::add contract); returns the number of output nodes
int oracle_add(double prec, void* out, int n, const double* c, void* const* f, int max_iter) {
    std::vector<double> cv(c, c + n);
    std::vector<const Tree*> fv;
    for (int i = 0; i < n; ++i) fv.push_back((const Tree*)f[i]);
    add(prec, *(Tree*)out, cv, fv, max_iter);
    return (int)((Tree*)out)->nodes.size();
}
// out = d/dx_dir inp on the input's grid (ABGV first derivative, flux parameters a, b)
int oracle_derivative(void* out, void* inp, double a, double b, int dir) {
    derivative_apply(*(Tree*)out, *(Tree*)inp, a, b, dir);
    return (int)((Tree*)out)->nodes.size();
}
// union of grids (mrcpp::build_grid contract); returns the number of nodes of `out`
int oracle_build_grid(void* out, void* inp) {
    build_grid(*(Tree*)out, *(Tree*)inp);
    return (int)((Tree*)out)->nodes.size();
}

int oracle_num_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
}
