import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a library")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O

    O.lib()
    return O


@pytest.fixture(scope="session")
def gpu_mod():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mrchem_b200 import mrcpp as G

    G.load_library()
    return G
