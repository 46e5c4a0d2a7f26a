"""B200-native multiwavelet operator apply (the MRCPP ``apply`` path behind MRChem).

The compute path is ``libmwb200.so`` (hand-written sm_100a kernels behind a C-ABI, declared in
``include/mwb200.h``); :mod:`mrchem_b200.mrcpp` is its Python mirror.
"""
from . import mrcpp  # noqa: F401

__all__ = ["mrcpp"]
