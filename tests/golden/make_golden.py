"""Regenerate tests/golden/oracle_small.npz: a small Poisson apply through the FP64 oracle
(order 5, prec 1e-3, one normalised Gaussian, exponent 10, centre (0.1,-0.2,0.3)), recording the
output node keys and squared norm.  Run: python tests/golden/make_golden.py"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import oracle as O  # noqa: E402


def main():
    m = O.MultiResolutionAnalysis(-2, (-5, -5, -5), (10, 10, 10), 5, 10)
    alpha = 10.0
    ftype, params = O.gauss_params([(alpha / np.pi) ** 1.5], [alpha], [(0.1, -0.2, 0.3)])
    inp = O.FunctionTree(m)
    O.project(1e-3, inp, (ftype, params))
    out = O.FunctionTree(m)
    O.apply(1e-3, out, O.PoissonOperator(m, 1e-3), inp)
    ex = out.export()
    keys = np.array(sorted((int(d), *map(int, t)) for d, t in zip(ex["depth"], ex["trans"])))
    np.savez(os.path.join(HERE, "oracle_small.npz"), ftype=ftype, params=params, out_keys=keys,
             out_norm2=out.square_norm())
    print(len(keys), out.square_norm())


if __name__ == "__main__":
    main()
