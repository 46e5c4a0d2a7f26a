"""The C-ABI library loads and exports every symbol include/*.h declares (CPU only: no compute calls)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(inc, fn)).read()
        if 'extern "C"' not in src:
            continue
        names |= set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s*(mw_[a-z0-9_]+)\s*\(", src, re.M))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert {"mw_apply", "mw_op_create_poisson", "mw_op_create_helmholtz", "mw_project", "mw_tree_upload"} <= names


def test_library_exports_every_declared_symbol():
    from mrchem_b200 import mrcpp

    lib = mrcpp.load_library()
    for name in sorted(declared_symbols()):
        assert hasattr(lib, name), name
    bound = {s[0] for s in mrcpp.SYMBOLS}
    assert declared_symbols() <= bound


def test_library_rejects_bad_arguments_without_gpu():
    """Argument checks run before any CUDA call and report through mw_last_error."""
    from mrchem_b200 import mrcpp

    lib = mrcpp.load_library()
    assert lib.mw_apply(1e-3, None, None, None, 0) != 0
    assert b"null" in lib.mw_last_error()
    assert lib.mw_tree_nnodes(None, None) != 0
    major, minor = ctypes.c_int(), ctypes.c_int()
    assert lib.mw_version(ctypes.byref(major), ctypes.byref(minor)) == 0
    assert (major.value, minor.value) >= (0, 1)


def test_oracle_library_loads():
    from oracle import oracle as O

    assert O.lib().oracle_num_threads() >= 1


def test_product_does_not_reference_oracle():
    """The product package never imports or links the oracle."""
    pkg = os.path.join(ROOT, "mrchem_b200")
    for dirpath, _, files in os.walk(pkg):
        for fn in files:
            if fn.endswith((".py", ".cu", ".cuh", ".hpp", ".cpp", ".h")) or fn == "Makefile":
                src = open(os.path.join(dirpath, fn), errors="ignore").read()
                for pat in (r"import\s+oracle", r"from\s+oracle", r"libmworacle", r"\boracle_[a-z_]+\s*\(", r"mw_oracle"):
                    assert not re.search(pat, src), (fn, pat)
