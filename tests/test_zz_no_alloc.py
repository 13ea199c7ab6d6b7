"""The no-allocation plain search entry point, called through the C ABI.

e8qc_e8q_search_plain_noalloc exists for callers that cannot let a search
allocate device memory (a framework that owns all of HBM through its caching
allocator, a request handler that must not be stalled by cudaFree's device
synchronisation, a JNI/cgo host with a fixed memory budget). It must return
what the regular plain search returns, call after call, since every call
reuses the same static scratch array. This file is collected last so a run
that stops at the first failure has already run every other test.
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import PKG
from gen import det_mixture
from parity import assert_topk_parity

pytestmark = pytest.mark.gpu


def _lib():
    lib = ctypes.CDLL(os.path.join(PKG, "e8qlib", "libe8qcuda.so"))
    vp, sz = ctypes.c_void_p, ctypes.c_size_t
    lib.e8qc_e8q_create.argtypes = [ctypes.c_int, sz, ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(vp)]
    lib.e8qc_e8q_build.argtypes = [vp, vp, sz, vp, sz, vp, ctypes.c_float, vp]
    lib.e8qc_e8q_search.argtypes = [vp, vp, sz, sz, sz, ctypes.c_int, vp, vp, vp, vp]
    lib.e8qc_e8q_search_plain_noalloc.argtypes = [vp, vp, sz, sz, sz, vp, vp, vp]
    lib.e8qc_e8q_destroy.argtypes = [vp]
    lib.e8qc_last_error.restype = ctypes.c_char_p
    return lib


def _ok(lib, rc):
    assert rc == 0, lib.e8qc_last_error().decode()


def test_noalloc_matches_plain_search_twice():
    import torch

    lib = _lib()
    dim, bits, nlist, n, nq, k, nprobe = 200, 5, 24, 5000, 37, 16, 6
    x, cm, lab = det_mixture(71, n, dim, nlist, 0.5)
    q = det_mixture(72, nq, dim, nlist, 0.5)[0]
    idx = ctypes.c_void_p()
    _ok(lib, lib.e8qc_e8q_create(0, dim, bits, 3, ctypes.byref(idx)))
    try:
        _ok(lib, lib.e8qc_e8q_build(idx, x.ctypes.data, n, cm.ctypes.data, nlist, lab.ctypes.data, 0.0, None))
        dev = torch.device("cuda", 0)
        qd = torch.from_numpy(q).to(dev)
        ref_ids = torch.empty(nq, k, dtype=torch.int32, device=dev)
        ref_d = torch.empty(nq, k, dtype=torch.float32, device=dev)
        torch.cuda.synchronize()
        _ok(lib, lib.e8qc_e8q_search(idx, qd.data_ptr(), nq, k, nprobe, 0, ref_ids.data_ptr(), ref_d.data_ptr(),
                                     None, None))
        want_ids = ref_ids.cpu().numpy().view(np.uint32)
        want_d = ref_d.cpu().numpy()
        for call in range(2):
            ids = torch.full((nq, k), -1, dtype=torch.int32, device=dev)
            d = torch.full((nq, k), -1.0, dtype=torch.float32, device=dev)
            torch.cuda.synchronize()
            _ok(lib, lib.e8qc_e8q_search_plain_noalloc(idx, qd.data_ptr(), nq, k, nprobe, ids.data_ptr(),
                                                       d.data_ptr(), None))
            assert_topk_parity(ids.cpu().numpy().view(np.uint32), d.cpu().numpy(), want_ids, want_d)
        # limits and argument checks fail loudly instead of allocating
        assert lib.e8qc_e8q_search_plain_noalloc(idx, qd.data_ptr(), nq, 0, nprobe, ids.data_ptr(),
                                                 d.data_ptr(), None) != 0
        host_ids = np.zeros((nq, k), np.uint32)
        assert lib.e8qc_e8q_search_plain_noalloc(idx, qd.data_ptr(), nq, k, nprobe, host_ids.ctypes.data,
                                                 d.data_ptr(), None) != 0
        assert b"device pointers" in lib.e8qc_last_error()
    finally:
        lib.e8qc_e8q_destroy(idx)
