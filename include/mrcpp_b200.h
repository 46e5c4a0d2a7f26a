// mrcpp_b200.h -- C++ front-end with the MRCPP names that the reference (MRChem) calls on the
// operator-apply path, implemented over the C-ABI of mwb200.h.  Header only; link libmwb200.so.
//
// The call sites compile unchanged against these declarations:
//   mrcpp::BoundingBox<3> world(min_scale, corner, boxes);              src/mrenv.cpp:52
//   mrcpp::InterpolatingBasis basis(order);                             src/mrenv.cpp:65
//   mrcpp::MultiResolutionAnalysis<3> MRA(world, basis, max_depth);     src/mrenv.cpp:66
//   mrcpp::FunctionTree<3> tree(MRA);                                   src/qmfunctions/QMFunction.cpp:71
//   mrcpp::PoissonOperator P(MRA, prec);                                src/SCFDriver.cpp:279
//   mrcpp::HelmholtzOperator H(MRA, mu, prec);                          src/scf_solver/HelmholtzVector.cpp:171
//   mrcpp::apply(prec, out, H, inp);                                    src/scf_solver/HelmholtzVector.cpp:176
//   tree.getSquareNorm(); tree.getNNodes(); tree.rescale(c);            src/scf_solver/HelmholtzVector.cpp:81-89
// Errors abort with a message, as MRCPP's MSG_FATAL does (the C-ABI itself returns status codes).
#ifndef MRCPP_B200_H
#define MRCPP_B200_H

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include "mwb200.h"

namespace mrcpp {

constexpr double MachineZero = 1.0e-14;

namespace detail {
inline void check(int status, const char* what) {
    if (status != MW_OK) {
        std::fprintf(stderr, "Error: %s failed (%d): %s\n", what, status, mw_last_error());
        std::abort();
    }
}
// one device context per process (device from MWB200_DEVICE, default 0)
inline mw_ctx context() {
    static mw_ctx ctx = [] {
        const char* e = std::getenv("MWB200_DEVICE");
        mw_ctx c = nullptr;
        check(mw_ctx_create(e ? std::atoi(e) : 0, nullptr, &c), "mw_ctx_create");
        return c;
    }();
    return ctx;
}
}  // namespace detail

template <int D> class BoundingBox;
template <> class BoundingBox<3> {
public:
    BoundingBox(int min_scale, const int* corner, const int* boxes) : scale_(min_scale) {
        for (int d = 0; d < 3; ++d) {
            corner_[d] = corner[d];
            boxes_[d] = boxes[d];
        }
    }
    int getScale() const { return scale_; }
    const int* getCornerIndex() const { return corner_; }
    const int* getNBoxes() const { return boxes_; }

private:
    int scale_;
    int corner_[3];
    int boxes_[3];
};

class ScalingBasis {
public:
    ScalingBasis(int type, int order) : type_(type), order_(order) {}
    int getScalingType() const { return type_; }
    int getScalingOrder() const { return order_; }

private:
    int type_, order_;
};
class InterpolatingBasis : public ScalingBasis {
public:
    explicit InterpolatingBasis(int order) : ScalingBasis(MW_BASIS_INTERPOLATING, order) {}
};
class LegendreBasis : public ScalingBasis {
public:
    explicit LegendreBasis(int order) : ScalingBasis(MW_BASIS_LEGENDRE, order) {}
};

template <int D> class MultiResolutionAnalysis;
template <> class MultiResolutionAnalysis<3> {
public:
    MultiResolutionAnalysis(const BoundingBox<3>& world, const ScalingBasis& basis, int max_depth)
            : order_(basis.getScalingOrder()), max_depth_(max_depth) {
        mw_mra h = nullptr;
        detail::check(mw_mra_create(detail::context(), world.getScale(), world.getCornerIndex(), world.getNBoxes(),
                                    basis.getScalingType(), basis.getScalingOrder(), max_depth, &h),
                      "MultiResolutionAnalysis");
        h_ = std::shared_ptr<mw_mra_s>(h, [](mw_mra p) { mw_mra_destroy(p); });
    }
    int getOrder() const { return order_; }
    int getMaxDepth() const { return max_depth_; }
    mw_mra handle() const { return h_.get(); }

private:
    int order_, max_depth_;
    std::shared_ptr<mw_mra_s> h_;
};

template <int D> class FunctionTree;
template <> class FunctionTree<3> {
public:
    explicit FunctionTree(const MultiResolutionAnalysis<3>& mra) : mra_(&mra) {
        detail::check(mw_tree_create(mra.handle(), &h_), "FunctionTree");
    }
    ~FunctionTree() { mw_tree_destroy(h_); }
    FunctionTree(const FunctionTree&) = delete;
    FunctionTree& operator=(const FunctionTree&) = delete;

    int getNNodes() const {
        int n = 0;
        detail::check(mw_tree_nnodes(h_, &n), "getNNodes");
        return n;
    }
    double getSquareNorm() const {
        double v = 0.0;
        detail::check(mw_tree_square_norm(h_, &v), "getSquareNorm");
        return v;
    }
    void rescale(double c) { detail::check(mw_tree_rescale(h_, c), "rescale"); }
    const MultiResolutionAnalysis<3>& getMRA() const { return *mra_; }
    mw_tree handle() const { return h_; }
    // checkpoint files (reference src/qmfunctions/Orbital.cpp:128,170)
    void saveTree(const std::string& file) { detail::check(mw_tree_save(h_, file.c_str()), "saveTree"); }
    void loadTree(const std::string& file) { detail::check(mw_tree_load(h_, file.c_str()), "loadTree"); }

private:
    const MultiResolutionAnalysis<3>* mra_;
    mw_tree h_ = nullptr;
};

// Sum of Cartesian Gaussians c (x-X)^px (y-Y)^py (z-Z)^pz exp(-alpha |r-R|^2) (GaussExp<3> analogue,
// the form in which MRChem's initial guesses are projected: src/initial_guess/gto.cpp:132-170).
template <int D> class GaussExp;
template <> class GaussExp<3> {
public:
    void append(double coef, double alpha, const double* pos, const int* pow = nullptr) {
        p_.push_back(coef);
        p_.push_back(alpha);
        for (int d = 0; d < 3; ++d) p_.push_back(pos[d]);
        for (int d = 0; d < 3; ++d) p_.push_back(pow ? pow[d] : 0);
        ++n_;
    }
    int size() const { return n_; }
    std::vector<double> params() const {
        std::vector<double> v{double(n_)};
        v.insert(v.end(), p_.begin(), p_.end());
        return v;
    }

private:
    int n_ = 0;
    std::vector<double> p_;
};

template <int D> class ConvolutionOperator;
template <> class ConvolutionOperator<3> {
public:
    virtual ~ConvolutionOperator() { mw_op_destroy(h_); }
    ConvolutionOperator(const ConvolutionOperator&) = delete;
    ConvolutionOperator& operator=(const ConvolutionOperator&) = delete;
    int size() const {
        int n = 0;
        detail::check(mw_op_nterms(h_, &n), "ConvolutionOperator::size");
        return n;
    }
    mw_op handle() const { return h_; }

protected:
    ConvolutionOperator() = default;
    mw_op h_ = nullptr;
};

// kernel 1/|r|
class PoissonOperator : public ConvolutionOperator<3> {
public:
    PoissonOperator(const MultiResolutionAnalysis<3>& mra, double prec) {
        detail::check(mw_op_create_poisson(mra.handle(), prec, &h_), "PoissonOperator");
    }
};

// kernel exp(-mu |r|)/|r|
class HelmholtzOperator : public ConvolutionOperator<3> {
public:
    HelmholtzOperator(const MultiResolutionAnalysis<3>& mra, double mu, double prec) {
        detail::check(mw_op_create_helmholtz(mra.handle(), mu, prec, &h_), "HelmholtzOperator");
    }
};

// first derivative with flux parameters a, b (reference src/SCFDriver.cpp:282-283)
template <int D> class DerivativeOperator;
template <> class DerivativeOperator<3> {
public:
    DerivativeOperator(const DerivativeOperator&) = delete;
    DerivativeOperator& operator=(const DerivativeOperator&) = delete;
    ~DerivativeOperator() {
        if (h_) mw_op_destroy(h_);
    }
    mw_op handle() const { return h_; }

protected:
    DerivativeOperator() = default;
    mw_op h_ = nullptr;
};
template <int D> class ABGVOperator;
template <> class ABGVOperator<3> : public DerivativeOperator<3> {
public:
    ABGVOperator(const MultiResolutionAnalysis<3>& mra, double a, double b) {
        detail::check(mw_op_create_abgv(mra.handle(), a, b, &h_), "ABGVOperator");
    }
};
// out = d/dx_dir inp on the input's grid (reference NablaOperator.cpp:35)
template <int D> void apply(FunctionTree<D>& out, DerivativeOperator<D>& op, FunctionTree<D>& inp, int dir);
template <> inline void apply<3>(FunctionTree<3>& out, DerivativeOperator<3>& op, FunctionTree<3>& inp, int dir) {
    detail::check(mw_apply_derivative(out.handle(), op.handle(), inp.handle(), dir, MW_APPLY_FP64), "apply");
}

// out = op * inp, adaptive to relative precision prec
template <int D> void apply(double prec, FunctionTree<D>& out, ConvolutionOperator<D>& op, FunctionTree<D>& inp);
template <> inline void apply<3>(double prec, FunctionTree<3>& out, ConvolutionOperator<3>& op, FunctionTree<3>& inp) {
    detail::check(mw_apply(prec, out.handle(), op.handle(), inp.handle(), MW_APPLY_FP64), "apply");
}

// adaptive projection of a Gaussian sum
inline void project(double prec, FunctionTree<3>& tree, const GaussExp<3>& f) {
    std::vector<double> p = f.params();
    detail::check(mw_project(prec, tree.handle(), MW_FUNC_GAUSSIANS, (int)p.size(), p.data()), "project");
}

inline double dot(FunctionTree<3>& a, FunctionTree<3>& b) {
    double v = 0.0;
    detail::check(mw_dot(a.handle(), b.handle(), &v), "dot");
    return v;
}

// out = c a b (reference call sites src/qmfunctions/qmfunction_utils.cpp:214,217); maxIter < 0 refines
// until converged, 0 keeps the grid of `out`
inline void multiply(double prec, FunctionTree<3>& out, double c, FunctionTree<3>& a, FunctionTree<3>& b,
                     int maxIter = -1) {
    detail::check(mw_multiply(prec, out.handle(), c, a.handle(), b.handle(), maxIter), "multiply");
}

// out = a^2 (reference src/qmfunctions/density_utils.cpp:74)
inline void square(double prec, FunctionTree<3>& out, FunctionTree<3>& a, int maxIter = -1) {
    detail::check(mw_square(prec, out.handle(), a.handle(), maxIter), "square");
}

// out = sum_i c_i f_i over (c_i, f_i) pairs (reference qmfunction_utils.cpp:170-177, KAIN.cpp:180)
template <int D> using FunctionTreeVector = std::vector<std::tuple<double, FunctionTree<D>*>>;
inline void add(double prec, FunctionTree<3>& out, FunctionTreeVector<3>& vec, int maxIter = -1) {
    std::vector<double> c;
    std::vector<mw_tree> f;
    for (auto& t : vec) {
        c.push_back(std::get<0>(t));
        f.push_back(std::get<1>(t)->handle());
    }
    detail::check(mw_add(prec, out.handle(), (int)f.size(), c.data(), f.data(), maxIter), "add");
}
// out = a A + b B
inline void add(double prec, FunctionTree<3>& out, double a, FunctionTree<3>& A, double b, FunctionTree<3>& B,
                int maxIter = -1) {
    FunctionTreeVector<3> vec{{a, &A}, {b, &B}};
    add(prec, out, vec, maxIter);
}

// grid helpers (reference qmfunction_utils.cpp:211-212, density_utils.cpp:73)
inline void build_grid(FunctionTree<3>& out, FunctionTree<3>& inp) {
    detail::check(mw_tree_build_grid(out.handle(), inp.handle()), "build_grid");
}
inline void copy_grid(FunctionTree<3>& out, FunctionTree<3>& inp) {
    detail::check(mw_tree_copy_grid(out.handle(), inp.handle()), "copy_grid");
}

}  // namespace mrcpp

#endif  // MRCPP_B200_H
