"""The C++ front-end (include/mrcpp_b200.h) compiles with the reference's call-site shapes and gives
the same results as the Python mirror of the C-ABI."""
import os
import re
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_frontend_matches_python(gpu_mod, tmp_path):
    G = gpu_mod
    exe = tmp_path / "helmholtz_apply"
    libdir = os.path.join(ROOT, "mrchem_b200")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", "helmholtz_apply.cpp"), "-L" + libdir, "-lmwb200",
                           "-Wl,-rpath," + libdir, "-o", str(exe)])
    env = dict(os.environ, MWB200_CKPT=str(tmp_path / "out_h.tree"))
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True, env=env).stdout
    vals = {}
    for line in out.splitlines():
        m = re.match(r"(\w+) nodes (\d+) norm2 (\S+) dot (\S+)", line)
        vals[m.group(1)] = (int(m.group(2)), float(m.group(3)), float(m.group(4)))

    m = G.MultiResolutionAnalysis(-2, (-5, -5, -5), (10, 10, 10), 7, 14)
    prec, alpha = 1e-5, 3.0
    phi = G.FunctionTree(m)
    G.project(prec, phi, G.gauss_params([(2 * alpha / np.pi) ** 0.75], [alpha], [(0.1, -0.2, 0.3)]))
    out_h = G.FunctionTree(m)
    G.apply(prec, out_h, G.HelmholtzOperator(m, 1.0, prec), phi)
    out_h.rescale(-1.0 / (2 * np.pi))
    V = G.FunctionTree(m)
    G.apply(prec / np.sqrt(phi.square_norm()), V, G.PoissonOperator(m, prec), phi)
    P = G.PoissonOperator(m, prec)
    phi_ip = G.FunctionTree(m)
    G.build_grid(phi_ip, phi)
    G.build_grid(phi_ip, out_h)
    G.multiply(-1.0, phi_ip, 1.0, phi, out_h, 0)
    V_ip = G.FunctionTree(m)
    G.apply(prec, V_ip, P, phi_ip)
    rho = G.FunctionTree(m)
    G.copy_grid(rho, phi)
    G.square(prec, rho, phi)
    arg = G.FunctionTree(m)
    G.add(prec, arg, [1.0, -2.0], [out_h, phi])
    dphi = G.FunctionTree(m)
    G.apply_derivative(dphi, G.ABGVOperator(m, 0.5, 0.5), phi, 1)
    for key, t in (("helmholtz", out_h), ("poisson", V), ("exchange", V_ip), ("density", rho), ("sum", arg),
                   ("derivative", dphi), ("checkpoint", out_h)):
        n, n2, d = vals[key]
        assert n == t.nnodes()
        assert abs(n2 - t.square_norm()) <= 1e-12 * t.square_norm()
        assert abs(d - G.dot(t, phi)) <= 1e-12 * abs(d)
