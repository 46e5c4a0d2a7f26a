"""Tree byte images (checkpoint files and inter-process payloads; FunctionTree::saveTree/loadTree,
reference src/qmfunctions/Orbital.cpp:118-190, and mrcpp::send_tree, src/parallel.cpp:208-232):
round trips are bit-exact, a different world or a damaged image is refused, and an image crosses a
process boundary (written by one process, read by another)."""
import os
import subprocess
import sys

import numpy as np
import pytest

from test_gpu_parity import WORLD, two_gaussians

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def same(a, b):
    ea, eb = a.export(), b.export()
    return all(np.array_equal(ea[k], eb[k]) for k in ("depth", "trans", "parent", "child0", "coef"))


def test_serialize_roundtrip_and_file(gpu_mod, tmp_path):
    G = gpu_mod
    m = G.MultiResolutionAnalysis(*WORLD, 7, 14)
    a = G.FunctionTree(m)
    G.project(1e-5, a, two_gaussians(G))
    img = a.serialize()
    assert img[:8].tobytes() == b"MWB2TREE"
    b = G.FunctionTree(m)
    b.deserialize(img)
    assert same(a, b) and b.square_norm() == a.square_norm()
    path = tmp_path / "phi_0_re.tree"
    a.save_tree(path)
    c = G.FunctionTree(m)
    c.load_tree(path)
    assert same(a, c)
    other = G.MultiResolutionAnalysis(*WORLD, 5, 14)
    with pytest.raises(G.MWError):
        G.FunctionTree(other).deserialize(img)  # other basis order
    bad = img.copy()
    bad[0] = ord("X")
    with pytest.raises(G.MWError):
        b.deserialize(bad)
    with pytest.raises(G.MWError):
        b.deserialize(img[: img.size // 2])


def test_image_crosses_processes(gpu_mod, tmp_path):
    """one process applies and checkpoints, another loads the file and gets the same tree"""
    G = gpu_mod
    m = G.MultiResolutionAnalysis(*WORLD, 7, 14)
    a = G.FunctionTree(m)
    G.project(1e-5, a, two_gaussians(G))
    v = G.FunctionTree(m)
    G.apply(1e-5, v, G.PoissonOperator(m, 1e-5), a)
    path = tmp_path / "v.tree"
    v.save_tree(path)
    code = f"""
import sys
sys.path.insert(0, {ROOT!r})
from mrchem_b200 import mrcpp as G
m = G.MultiResolutionAnalysis(-2, (-5, -5, -5), (10, 10, 10), 7, 14)
t = G.FunctionTree(m)
t.load_tree({str(path)!r})
print(t.nnodes(), repr(t.square_norm()))
"""
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True).stdout.split()
    assert int(out[0]) == v.nnodes() and float(out[1]) == v.square_norm()
