"""The no-allocation plain search entry point, called through the C ABI.

e8qc_e8q_search_plain_noalloc exists for callers that cannot let a search
allocate device memory (a framework that owns all of HBM through its caching
allocator, a request handler that must not be stalled by cudaFree's device
synchronisation, a JNI/cgo host with a fixed memory budget). It must return
what the oracle and the regular plain search return, call after call, since
every call reuses the same static scratch array, and it must leave the
device's free memory as it found it. This file is collected last so a run
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

EINVAL = -1


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


class _Index:
    """A device index built through the C ABI (destroyed on exit)."""

    def __init__(self, lib, x, cm, lab, bits, seed):
        self.lib = lib
        self.p = ctypes.c_void_p()
        n, dim = x.shape
        _ok(lib, lib.e8qc_e8q_create(0, dim, bits, seed, ctypes.byref(self.p)))
        _ok(lib, lib.e8qc_e8q_build(self.p, x.ctypes.data, n, cm.ctypes.data, cm.shape[0], lab.ctypes.data,
                                    0.0, None))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.lib.e8qc_e8q_destroy(self.p)


def _noalloc(lib, idx, qd, k, nprobe, stream=None):
    import torch

    nq = qd.shape[0]
    ids = torch.full((nq, k), -1, dtype=torch.int32, device=qd.device)
    d = torch.full((nq, k), -1.0, dtype=torch.float32, device=qd.device)
    torch.cuda.synchronize()
    _ok(lib, lib.e8qc_e8q_search_plain_noalloc(idx.p, qd.data_ptr(), nq, k, nprobe, ids.data_ptr(), d.data_ptr(),
                                               None if stream is None else stream.cuda_stream))
    return ids.cpu().numpy().view(np.uint32), d.cpu().numpy()


def _plain(lib, idx, qd, k, nprobe):
    import torch

    nq = qd.shape[0]
    ids = torch.empty(nq, k, dtype=torch.int32, device=qd.device)
    d = torch.empty(nq, k, dtype=torch.float32, device=qd.device)
    torch.cuda.synchronize()
    _ok(lib, lib.e8qc_e8q_search(idx.p, qd.data_ptr(), nq, k, nprobe, 0, ids.data_ptr(), d.data_ptr(), None, None))
    torch.cuda.synchronize()
    return ids.cpu().numpy().view(np.uint32), d.cpu().numpy()


@pytest.mark.parametrize("shape", [
    # dim, bits, nlist, n, nq, k, nprobe
    (200, 5, 24, 5000, 37, 16, 6),
    # more than 1,024 probed lists (tile offsets read from global memory) and k = 128
    (64, 4, 1100, 20000, 9, 128, 1100),
])
def test_noalloc_matches_oracle_and_plain_twice(oracle_lib, shape):
    """Two calls in a row equal the oracle's search and the regular plain
    search, and neither call changes the device's free memory."""
    import torch

    dim, bits, nlist, n, nq, k, nprobe = shape
    lib = _lib()
    x, cm, lab = det_mixture(71, n, dim, nlist, 0.5)
    q = det_mixture(72, nq, dim, nlist, 0.5)[0]
    orc = oracle_lib.OracleE8qIndex(x, cm, lab, bits, seed=3, threads=8)
    ref_ids, ref_d = orc.search(q, k, nprobe, threads=8)
    with _Index(lib, x, cm, lab, bits, 3) as idx:
        dev = torch.device("cuda", 0)
        qd = torch.from_numpy(q).to(dev)
        want_ids, want_d = _plain(lib, idx, qd, k, nprobe)
        assert_topk_parity(want_ids, want_d, ref_ids, ref_d)
        _noalloc(lib, idx, qd, k, nprobe)  # the first call on the device resolves the scratch address
        for call in range(2):
            # result buffers exist before the free-memory reading
            ids = torch.full((nq, k), -1, dtype=torch.int32, device=dev)
            d = torch.full((nq, k), -1.0, dtype=torch.float32, device=dev)
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info(0)[0]
            _ok(lib, lib.e8qc_e8q_search_plain_noalloc(idx.p, qd.data_ptr(), nq, k, nprobe, ids.data_ptr(),
                                                       d.data_ptr(), None))
            torch.cuda.synchronize()
            free1 = torch.cuda.mem_get_info(0)[0]
            assert free1 == free0, f"call {call}: device free memory changed by {free0 - free1} bytes"
            got_ids, got_d = ids.cpu().numpy().view(np.uint32), d.cpu().numpy()
            assert_topk_parity(got_ids, got_d, ref_ids, ref_d)
            assert_topk_parity(got_ids, got_d, want_ids, want_d)


def test_noalloc_on_a_stream_and_argument_checks():
    import torch

    lib = _lib()
    dim, bits, nlist, n, nq, k, nprobe = 96, 6, 16, 3000, 11, 10, 5
    x, cm, lab = det_mixture(81, n, dim, nlist, 0.5)
    q = det_mixture(82, nq, dim, nlist, 0.5)[0]
    with _Index(lib, x, cm, lab, bits, 5) as idx:
        dev = torch.device("cuda", 0)
        qd = torch.from_numpy(q).to(dev)
        want_ids, want_d = _plain(lib, idx, qd, k, nprobe)
        st = torch.cuda.Stream(device=dev)
        for _ in range(2):
            got_ids, got_d = _noalloc(lib, idx, qd, k, nprobe, stream=st)
            assert_topk_parity(got_ids, got_d, want_ids, want_d)
        ids = torch.empty(nq, k, dtype=torch.int32, device=dev)
        d = torch.empty(nq, k, dtype=torch.float32, device=dev)
        # bad arguments fail loudly instead of allocating or launching
        assert lib.e8qc_e8q_search_plain_noalloc(idx.p, qd.data_ptr(), nq, 0, nprobe, ids.data_ptr(),
                                                 d.data_ptr(), None) == EINVAL
        assert lib.e8qc_e8q_search_plain_noalloc(idx.p, qd.data_ptr(), nq, 129, nprobe, ids.data_ptr(),
                                                 d.data_ptr(), None) == EINVAL
        assert lib.e8qc_e8q_search_plain_noalloc(idx.p, qd.data_ptr(), nq, k, 0, ids.data_ptr(),
                                                 d.data_ptr(), None) == EINVAL
        host_ids = np.zeros((nq, k), np.uint32)
        assert lib.e8qc_e8q_search_plain_noalloc(idx.p, qd.data_ptr(), nq, k, nprobe, host_ids.ctypes.data,
                                                 d.data_ptr(), None) == EINVAL
        assert b"device pointers" in lib.e8qc_last_error()
        if torch.cuda.device_count() > 1:
            # a result buffer on another GPU is refused, not dereferenced
            other = torch.empty(nq, k, dtype=torch.int32, device=torch.device("cuda", 1))
            assert lib.e8qc_e8q_search_plain_noalloc(idx.p, qd.data_ptr(), nq, k, nprobe, other.data_ptr(),
                                                     d.data_ptr(), None) == EINVAL


@pytest.mark.parametrize("case", ["padded_dim", "nlist"])
def test_noalloc_rejects_indexes_beyond_the_scratch_array(case):
    """Indexes the static array cannot serve are refused before any launch."""
    import torch

    lib = _lib()
    if case == "padded_dim":
        dim, nlist, n = 4100, 2, 64  # padded_dim 4160 > 4096
    else:
        dim, nlist, n = 8, 65537, 65537  # one vector per list, 65,537 lists > 65,536
    rng = np.random.default_rng(5)
    x = rng.standard_normal((n, dim), dtype=np.float32)
    lab = (np.arange(n) % nlist).astype(np.uint32)
    cm = np.zeros((nlist, dim), np.float32)
    np.add.at(cm, lab, x)
    cm /= np.maximum(np.bincount(lab, minlength=nlist), 1)[:, None].astype(np.float32)
    with _Index(lib, x, cm, lab, 4, 1) as idx:
        dev = torch.device("cuda", 0)
        qd = torch.from_numpy(x[:3].copy()).to(dev)
        ids = torch.empty(3, 10, dtype=torch.int32, device=dev)
        d = torch.empty(3, 10, dtype=torch.float32, device=dev)
        rc = lib.e8qc_e8q_search_plain_noalloc(idx.p, qd.data_ptr(), 3, 10, 4, ids.data_ptr(), d.data_ptr(), None)
        assert rc == EINVAL
        msg = lib.e8qc_last_error()
        assert (b"padded_dim" in msg) if case == "padded_dim" else (b"65536 lists" in msg)
