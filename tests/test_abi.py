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


def _plan_call(lib, fn, *args):
    cnt = ctypes.c_size_t()
    lens = (ctypes.c_size_t * 256)()
    bits = (ctypes.c_int * 256)()
    rc = fn(*args, lens, bits, 256, ctypes.byref(cnt))
    return rc, [(lens[i], bits[i]) for i in range(cnt.value)]


def test_me8q_host_plan_matches_oracle_and_golden(built, oracle_lib):
    """The library's host DP plan (e8qc_me8q_allocate) equals the oracle's on
    varied spectra and the reference's plans in the ME8Q fixtures; its plan
    parser accepts and rejects what the reference's does."""
    import numpy as np

    from conftest import load_golden
    from gen import det_mixture

    lib = ctypes.CDLL(os.path.join(PKG, "e8qlib", "libe8qcuda.so"))
    lib.e8qc_me8q_allocate.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_float, ctypes.c_int,
                                       ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                       ctypes.c_void_p]
    lib.e8qc_me8q_parse_plan.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_size_t, ctypes.c_void_p]
    rng = np.random.default_rng(5)
    cases = [(np.ones(256, np.float32), 4.0, 13, 0.0),
             (np.concatenate([np.linspace(4, 1, 192), np.zeros(64)]).astype(np.float32), 3.0, 13, 0.0),
             (np.zeros(128, np.float32), 2.0, 13, 0.0)]
    for pd in (64, 192, 512, 1024):
        for avg in (0.5, 1.0, 1.5, 2.0, 3.0, 4.5, 8.0):
            v = (rng.gamma(0.6, 1.0, pd) * np.exp(-np.arange(pd) / (pd / 3))).astype(np.float32)
            cases.append((v, avg, 13 if avg < 4 else 9, 0.0 if avg != 3.0 else 17.0))
    for v, avg, mb, extra in cases:
        rc, plan = _plan_call(lib, lib.e8qc_me8q_allocate, v.ctypes.data, v.shape[0], avg, mb, extra)
        assert rc == 0
        assert plan == [tuple(p) for p in oracle_lib.me8q_allocate(v, avg, mb, extra)], (v.shape, avg)
        assert sum(p[0] for p in plan) == v.shape[0]
    for name in ("me8q_d200_a4", "me8q_d150_a3", "me8q_d96_a6"):
        G = load_golden(name + ".npz")
        dim, seed, n, nlist = (int(t) for t in G["params"][:4])
        x = det_mixture(seed + 5000 + dim, n, dim, nlist, float(G["sigma"]))[0]
        pd = (dim + 63) // 64 * 64
        var = np.zeros(pd, np.float32)
        var[:dim] = oracle_lib.me8q_variance(x)
        rc, plan = _plan_call(lib, lib.e8qc_me8q_allocate, var.ctypes.data, pd, float(G["avg_bits"]), 13, 0.0)
        assert rc == 0 and plan == [tuple(p) for p in G["plan"]], name
    rc, plan = _plan_call(lib, lib.e8qc_me8q_parse_plan, b"64:6,64:4,,64:3,64:0", 256)
    assert rc == 0 and plan == [(64, 6), (64, 4), (64, 3), (64, 0)]
    for bad in (b"64:3", b"60:3,68:0", b"64-3,64:0", b"64:14,64:0", b"0:3,128:2"):
        rc, _ = _plan_call(lib, lib.e8qc_me8q_parse_plan, bad, 128)
        assert rc == -1, bad


def test_me8q_python_api_surface(built):
    import e8qlib

    cls = e8qlib.Me8qIndex
    for m in ("build", "search", "estimate", "export_codes"):
        assert hasattr(cls, m), m
    for p in ("dim", "avg_bits", "is_built", "n", "num_clusters", "bits_per_dim", "memory_bytes", "plan"):
        assert isinstance(getattr(cls, p), property), p
    idx = cls(200, 3.5, 9)
    assert idx.dim == 200 and idx.avg_bits == 3.5 and not idx.is_built and idx.n == 0 and idx.plan == []
    import numpy as np

    with pytest.raises(RuntimeError, match="built or loaded"):
        idx.search(np.zeros((1, 200), np.float32), 10, 4)
    with pytest.raises(RuntimeError, match="built or loaded"):
        idx.estimate(np.zeros(200, np.float32), 0)
    with pytest.raises(ValueError):
        cls(0, 4.0)
    with pytest.raises(ValueError):
        cls(16, 0.0)
