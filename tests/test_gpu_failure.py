"""Failure paths on the GPU, provoked without faulting, trapping or hanging
the device:

  * a bounded device wait that runs out (the scan kernel made to wait on a
    barrier nothing completes) returns E8QC_ETIMEOUT through the C ABI and
    raises in Python, within about its bound; the index stays usable and the
    next search returns exactly what it returned before;
  * a served request can be canceled while it waits for a batch slot, and a
    request that waits longer than request_timeout_ms expires; neither
    disturbs the other requests, whose results equal a search of the same
    queries alone;
  * an injected host-allocation failure at request intake is reported as out
    of memory and the server keeps serving.
"""
import ctypes
import os
import time

import numpy as np
import pytest

from conftest import PKG
from gen import det_mixture

pytestmark = pytest.mark.gpu

ETIMEOUT = -7


@pytest.fixture(scope="module")
def e8q():
    import e8qlib

    return e8qlib


@pytest.fixture(scope="module")
def index(e8q):
    dim = 128
    x, cm, lab = det_mixture(911, 40000, dim, 64, 0.5)
    idx = e8q.E8qIndex(dim, 4, 3)
    idx.build(x, cm, lab)
    q = det_mixture(912, 2048, dim, 64, 0.5)[0]
    return idx, q


def same(a, b):
    return np.array_equal(a[0], b[0]) and np.array_equal(np.asarray(a[1]).view(np.uint32),
                                                         np.asarray(b[1]).view(np.uint32))


def test_bounded_wait_timeout_is_reported_and_the_index_recovers(e8q, index):
    idx, q = index
    base = idx.search(q[:16], 10, 12, mode="plain")
    idx.debug_inject_wait_timeout(1, 50)
    t = time.perf_counter()
    with pytest.raises(RuntimeError, match="bounded device wait"):
        idx.search(q[:16], 10, 12, mode="plain")
    assert time.perf_counter() - t < 5.0  # gave up near its 50 ms bound, no hang
    assert same(idx.search(q[:16], 10, 12, mode="plain"), base)
    # several in a row, then normal again
    idx.debug_inject_wait_timeout(2, 20)
    for _ in range(2):
        with pytest.raises(RuntimeError):
            idx.search(q[:1], 10, 12, mode="plain")
    assert same(idx.search(q[:16], 10, 12, mode="plain"), base)
    idx.debug_inject_wait_timeout(3, 20)
    idx.debug_inject_wait_timeout(0, 0)  # cleared before any search ran
    assert same(idx.search(q[:16], 10, 12, mode="plain"), base)
    with pytest.raises(ValueError):
        idx.debug_inject_wait_timeout(1, 0)


def test_bounded_wait_timeout_through_the_c_abi(index):
    """The same, calling the library the way a C host would: the search
    returns E8QC_ETIMEOUT and the next one succeeds with the same rows."""
    lib = ctypes.CDLL(os.path.join(PKG, "e8qlib", "libe8qcuda.so"))
    vp, sz = ctypes.c_void_p, ctypes.c_size_t
    lib.e8qc_e8q_create.argtypes = [ctypes.c_int, sz, ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(vp)]
    lib.e8qc_e8q_build.argtypes = [vp, vp, sz, vp, sz, vp, ctypes.c_float, vp]
    lib.e8qc_e8q_search.argtypes = [vp, vp, sz, sz, sz, ctypes.c_int, vp, vp, vp, vp]
    lib.e8qc_e8q_debug_inject_wait_timeout.argtypes = [vp, ctypes.c_int, ctypes.c_uint32]
    lib.e8qc_e8q_destroy.argtypes = [vp]
    lib.e8qc_last_error.restype = ctypes.c_char_p
    x, cm, lab = det_mixture(77, 6000, 96, 24, 0.5)
    q = det_mixture(78, 8, 96, 24, 0.5)[0]
    p = vp()
    assert lib.e8qc_e8q_create(0, 96, 5, 1, ctypes.byref(p)) == 0
    try:
        assert lib.e8qc_e8q_build(p, x.ctypes.data, len(x), cm.ctypes.data, len(cm), lab.ctypes.data, 0.0,
                                  None) == 0
        rows = []
        for inject in (0, 1, 0):
            ids = np.zeros((8, 10), np.uint32)
            d = np.zeros((8, 10), np.float32)
            if inject:
                assert lib.e8qc_e8q_debug_inject_wait_timeout(p, 1, 30) == 0
            rc = lib.e8qc_e8q_search(p, q.ctypes.data, 8, 10, 6, 0, ids.ctypes.data, d.ctypes.data, None, None)
            if inject:
                assert rc == ETIMEOUT, lib.e8qc_last_error()
            else:
                assert rc == 0, lib.e8qc_last_error()
                rows.append((ids, d))
        assert same(rows[0], rows[1])
    finally:
        lib.e8qc_e8q_destroy(p)


def test_server_cancel(e8q, index):
    idx, q = index
    with e8q.Server(idx, mode="batched", max_batch=256, max_k=10, max_nprobe=64, slots=1) as srv:
        # a queue of full batches, then a small request behind them
        big = [srv.submit(q[256 * j:256 * (j + 1)], 10, 64) for j in range(6)]
        small = srv.submit(q[:4], 10, 8)
        srv.cancel(small)
        with pytest.raises(RuntimeError, match="canceled"):
            srv.result(small, timeout_ms=60000)
        for j, r in enumerate(big):
            got = srv.result(r, timeout_ms=60000)
            assert same(got, idx.search(q[256 * j:256 * (j + 1)], 10, 64, mode="batched"))
        with pytest.raises(IndexError):
            srv.cancel(small)  # already collected
        # canceling a request that already completed leaves its result
        r = srv.submit(q[:8], 10, 8)
        time.sleep(0.2)
        srv.cancel(r)
        got = srv.result(r, timeout_ms=60000)
        assert same(got, idx.search(q[:8], 10, 8, mode="batched"))
        st = srv.stats()
    assert st["canceled"] == 1
    assert st["completed"] == len(big) + 1


def test_server_request_timeout(e8q, index):
    idx, q = index
    with e8q.Server(idx, mode="batched", max_batch=256, max_k=10, max_nprobe=64, slots=1,
                    request_timeout_ms=1) as srv:
        reqs = [(q[(256 * j) % 2048:(256 * j) % 2048 + 256], srv.submit(q[(256 * j) % 2048:(256 * j) % 2048 + 256],
                                                                        10, 64)) for j in range(64)]
        done, expired = 0, 0
        for qq, r in reqs:
            try:
                got = srv.result(r, timeout_ms=60000)
            except RuntimeError as e:
                assert "expired" in str(e)
                expired += 1
                continue
            done += 1
            assert same(got, idx.search(qq, 10, 64, mode="batched"))
        st = srv.stats()
        # the first request is admitted at once; a 64-deep queue of full
        # batches keeps later ones waiting well past 1 ms
        assert done >= 1 and expired >= 1
        assert st["expired"] == expired and st["completed"] == done
        # the server keeps serving afterwards
        r = srv.submit(q[:4], 10, 8)
        assert same(srv.result(r, timeout_ms=60000), idx.search(q[:4], 10, 8, mode="batched"))


def test_server_host_allocation_failure(e8q, index):
    idx, q = index
    with e8q.Server(idx, mode="batched", max_batch=256, max_k=10, max_nprobe=64, slots=2) as srv:
        e8q.debug_fail_host_allocs(1)
        try:
            with pytest.raises(RuntimeError, match="out of memory"):
                srv.submit(q[:4], 10, 8)
        finally:
            e8q.debug_fail_host_allocs(0)
        r = srv.submit(q[:4], 10, 8)
        assert same(srv.result(r, timeout_ms=60000), idx.search(q[:4], 10, 8, mode="batched"))
        st = srv.stats()
    assert st["submitted"] == 1 and st["completed"] == 1
