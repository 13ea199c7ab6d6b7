"""CPU checks of the drop-in boundary: the C ABI library loads and exports
every entry point include/e8qc.h declares; the Python module imports and
mirrors the reference API surface. No compute calls (no GPU here)."""
import ctypes
import os
import re

import pytest

from conftest import PKG, ROOT


def _header_symbols():
    txt = open(os.path.join(ROOT, "include", "e8qc.h")).read()
    return sorted(set(re.findall(r"\b(e8qc_[a-z0-9_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def built():
    import sys

    sys.path.insert(0, PKG)
    import build as b

    b.build()
    return b


def test_library_exports_every_declared_symbol(built):
    lib = ctypes.CDLL(os.path.join(PKG, "e8qlib", "libe8qcuda.so"))
    syms = _header_symbols()
    assert len(syms) >= 17
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_version_and_codec_calls_without_gpu(built):
    lib = ctypes.CDLL(os.path.join(PKG, "e8qlib", "libe8qcuda.so"))
    assert lib.e8qc_version() >= 10000
    lib.e8qc_fixed_scale.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    s = ctypes.c_double()
    assert lib.e8qc_fixed_scale(4, ctypes.byref(s)) == 0 and abs(s.value - 0.785) < 1e-12
    lib.e8qc_last_error.restype = ctypes.c_char_p
    lib.e8qc_branch_levels.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    assert lib.e8qc_branch_levels(14, 0, None) == -1  # E8QC_EINVAL
    assert b"bits" in lib.e8qc_last_error()


def test_host_level_tables_match_golden(built):
    """The library's host-side level tables (used to build the GPU tables)
    equal the reference's, bit for bit."""
    import hashlib

    import numpy as np

    from conftest import load_golden

    lib = ctypes.CDLL(os.path.join(PKG, "e8qlib", "libe8qcuda.so"))
    lib.e8qc_branch_levels.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    g = load_golden("levels.npz")
    for b in range(1, 14):
        for br in (0, 1):
            a = np.zeros(1 << b, np.float64)
            assert lib.e8qc_branch_levels(b, br, a.ctypes.data) == 0
            assert hashlib.sha256(a.tobytes()).digest() == g[f"sha_b{b}_br{br}"].tobytes()


def test_python_module_api_surface(built):
    import e8qlib

    cls = e8qlib.E8qIndex
    for m in ("build", "search", "estimate", "set_disable_prune", "set_prune_alpha", "search_ragged",
              "search_ptr", "build_ptr", "export_codes"):
        assert hasattr(cls, m), m
    for p in ("dim", "nbits", "is_built", "n", "num_clusters", "memory_bytes", "disable_prune"):
        assert isinstance(getattr(cls, p), property), p
    idx = cls(96, 4, 3)
    assert idx.dim == 96 and idx.nbits == 4 and not idx.is_built and idx.n == 0
    import pytest as _pt

    with _pt.raises(ValueError):
        cls(16, 14)
