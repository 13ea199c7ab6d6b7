"""Failure paths made on the host, no GPU needed: an injected host-allocation
failure at index creation returns E8QC_ENOMEM (Python: "out of memory"),
changes nothing, and is consumed, so the next call proceeds normally."""
import ctypes
import os
import sys

import pytest

from conftest import PKG

ENOMEM = -4


@pytest.fixture(scope="module")
def lib():
    sys.path.insert(0, PKG)
    import build as b

    b.build()
    lib = ctypes.CDLL(os.path.join(PKG, "e8qlib", "libe8qcuda.so"))
    vp = ctypes.c_void_p
    lib.e8qc_e8q_create.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(vp)]
    lib.e8qc_me8q_create.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.c_float, ctypes.c_uint64,
                                     ctypes.POINTER(vp)]
    lib.e8qc_debug_fail_host_allocs.argtypes = [ctypes.c_int]
    lib.e8qc_last_error.restype = ctypes.c_char_p
    yield lib
    lib.e8qc_debug_fail_host_allocs(0)


def test_injected_host_allocation_failures_are_reported_and_consumed(lib):
    p = ctypes.c_void_p()
    assert lib.e8qc_debug_fail_host_allocs(2) == 0
    assert lib.e8qc_e8q_create(0, 64, 4, 0, ctypes.byref(p)) == ENOMEM
    assert b"host allocation failed" in lib.e8qc_last_error()
    assert not p.value  # nothing was created
    assert lib.e8qc_me8q_create(0, 64, 4.0, 0, ctypes.byref(p)) == ENOMEM
    assert not p.value
    # both injected failures are used up: the next call gets past the
    # allocation point (without a GPU it then stops at the device check)
    rc = lib.e8qc_e8q_create(0, 64, 4, 0, ctypes.byref(p))
    assert rc != ENOMEM
    if rc == 0:
        lib.e8qc_e8q_destroy.argtypes = [ctypes.c_void_p]
        lib.e8qc_e8q_destroy(p)
    assert lib.e8qc_debug_fail_host_allocs(-1) == -1  # E8QC_EINVAL


def test_python_surface_raises_out_of_memory(lib):
    """E8qIndex creates its native index in build(); an injected failure there
    surfaces as the "out of memory" RuntimeError before any device work."""
    import numpy as np

    import e8qlib

    x = np.zeros((64, 64), np.float32)
    cm = np.zeros((2, 64), np.float32)
    lab = np.zeros(64, np.uint32)
    e8qlib.debug_fail_host_allocs(1)
    try:
        with pytest.raises(RuntimeError, match="out of memory"):
            e8qlib.E8qIndex(64, 4, 0).build(x, cm, lab)
    finally:
        e8qlib.debug_fail_host_allocs(0)
