// Drop-in check of the C++ front-end: the calls below have the shapes of the reference's call sites
// (src/mrenv.cpp:52-66, src/scf_solver/HelmholtzVector.cpp:169-180, src/SCFDriver.cpp:279,
// src/qmoperators/two_electron/CoulombPotential.cpp:80-85, src/qmfunctions/qmfunction_utils.cpp:209-217,
// src/qmoperators/two_electron/ExchangePotential.cpp:131-137, src/qmfunctions/density_utils.cpp:73-74)
// and run on the GPU through libmwb200.so.
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "mrcpp_b200.h"

int main() {
    int min_scale = -2;
    int corner[3] = {-5, -5, -5};
    int boxes[3] = {10, 10, 10};
    mrcpp::BoundingBox<3> world(min_scale, corner, boxes);
    mrcpp::InterpolatingBasis basis(7);
    mrcpp::MultiResolutionAnalysis<3> MRA(world, basis, 14);

    const double prec = 1.0e-5;
    mrcpp::GaussExp<3> phi_f;  // a normalised Gaussian "orbital"
    const double alpha = 3.0, pos[3] = {0.1, -0.2, 0.3};
    phi_f.append(std::pow(2.0 * alpha / M_PI, 0.75), alpha, pos);
    mrcpp::FunctionTree<3> phi(MRA);
    mrcpp::project(prec, phi, phi_f);

    // HelmholtzVector::apply: mu = sqrt(-2 lambda), H(MRA, mu, prec), apply, rescale(-1/2pi)
    const double lambda = -0.5;
    const double mu = std::sqrt(-2.0 * lambda);
    mrcpp::HelmholtzOperator H(MRA, mu, prec);
    mrcpp::FunctionTree<3> out(MRA);
    mrcpp::apply(prec, out, H, phi);
    out.rescale(-1.0 / (2.0 * M_PI));
    std::printf("helmholtz nodes %d norm2 %.15e dot %.15e\n", out.getNNodes(), out.getSquareNorm(),
                mrcpp::dot(out, phi));

    // CoulombPotential::setupPotential: P(MRA, prec), abs_prec = prec / ||rho||, apply
    mrcpp::PoissonOperator P(MRA, prec);
    const double abs_prec = prec / std::sqrt(phi.getSquareNorm());
    mrcpp::FunctionTree<3> V(MRA);
    mrcpp::apply(abs_prec, V, P, phi);
    std::printf("poisson nodes %d norm2 %.15e dot %.15e\n", V.getNNodes(), V.getSquareNorm(), mrcpp::dot(V, phi));

    // ExchangePotential: phi_ip = phi_i^* phi_p on the union grid (multiply_real with prec < 0), then
    // V_ip = P[phi_ip]
    mrcpp::FunctionTree<3> phi_ip(MRA);
    mrcpp::build_grid(phi_ip, phi);
    mrcpp::build_grid(phi_ip, out);
    mrcpp::multiply(-1.0, phi_ip, 1.0, phi, out, 0);
    mrcpp::FunctionTree<3> V_ip(MRA);
    mrcpp::apply(prec, V_ip, P, phi_ip);
    std::printf("exchange nodes %d norm2 %.15e dot %.15e\n", V_ip.getNNodes(), V_ip.getSquareNorm(),
                mrcpp::dot(V_ip, phi));

    // density_utils::compute: copy_grid, then square
    mrcpp::FunctionTree<3> rho(MRA);
    mrcpp::copy_grid(rho, phi);
    mrcpp::square(prec, rho, phi);
    std::printf("density nodes %d norm2 %.15e dot %.15e\n", rho.getNNodes(), rho.getSquareNorm(), mrcpp::dot(rho, phi));

    // HelmholtzVector::apply's argument V phi + psi (HelmholtzVector.cpp:133-135): an adaptive sum
    mrcpp::FunctionTree<3> arg(MRA);
    mrcpp::add(prec, arg, 1.0, out, -2.0, phi);
    std::printf("sum nodes %d norm2 %.15e dot %.15e\n", arg.getNNodes(), arg.getSquareNorm(), mrcpp::dot(arg, phi));

    // QMNabla::apply: ABGVOperator<3>(MRA, 0.5, 0.5) along y (SCFDriver.cpp:283, NablaOperator.cpp:35)
    mrcpp::ABGVOperator<3> D(MRA, 0.5, 0.5);
    mrcpp::FunctionTree<3> dphi(MRA);
    mrcpp::apply(dphi, D, phi, 1);
    std::printf("derivative nodes %d norm2 %.15e dot %.15e\n", dphi.getNNodes(), dphi.getSquareNorm(), mrcpp::dot(dphi, phi));

    // Orbital::saveOrbital / loadOrbital (Orbital.cpp:128,170): checkpoint round trip
    const char* ckpt = std::getenv("MWB200_CKPT");
    if (ckpt) {
        out.saveTree(ckpt);
        mrcpp::FunctionTree<3> back(MRA);
        back.loadTree(ckpt);
        std::printf("checkpoint nodes %d norm2 %.15e dot %.15e\n", back.getNNodes(), back.getSquareNorm(), mrcpp::dot(back, phi));
    }
    return 0;
}
