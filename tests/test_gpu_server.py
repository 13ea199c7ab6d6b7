"""Serving loop (continuous batching over one index) on the GPU: every
request's result is bitwise the same as the same queries searched alone;
requests from several threads interleave; admission by memory splits the
stream into smaller batches without changing results; stats and errors."""
import threading

import numpy as np
import pytest

from gen import det_mixture

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def e8q():
    import e8qlib

    return e8qlib


@pytest.fixture(scope="module")
def index(e8q):
    dim, bits = 192, 6
    x, cm, lab = det_mixture(501, 8000, dim, 48, 0.5)
    idx = e8q.E8qIndex(dim, bits, 7)
    idx.build(x, cm, lab)
    q = det_mixture(502, 600, dim, 48, 0.5)[0]
    return idx, q


def make_requests(rng, q, n):
    reqs, off = [], 0
    for _ in range(n):
        m = int(rng.integers(1, 17))
        if off + m > len(q):
            off = 0
        reqs.append((q[off:off + m], int(rng.choice([1, 5, 10, 32, 100])), int(rng.integers(1, 49))))
        off += m
    return reqs


def same(a, b):
    return np.array_equal(a[0], b[0]) and np.array_equal(a[1].view(np.uint32), b[1].view(np.uint32))


@pytest.mark.parametrize("mode", ["precision", "batched"])
def test_server_matches_alone(e8q, index, mode):
    idx, q = index
    rng = np.random.default_rng(3)
    reqs = make_requests(rng, q, 80)
    with e8q.Server(idx, mode=mode, max_batch=256, slots=2) as srv:
        ids = [srv.submit(qq, k, npb) for qq, k, npb in reqs]
        got = [srv.result(i, timeout_ms=60000) for i in ids]
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["queries_completed"] == sum(len(r[0]) for r in reqs)
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    assert st["batches"] >= 1 and st["qps"] > 0
    for (qq, k, npb), res in zip(reqs, got):
        assert res is not None
        alone = idx.search(qq, k, npb, mode=mode)
        assert same(res, alone), (k, npb)


def test_server_threads_and_admission(e8q, index):
    """Four submitting threads; a memory budget that admits only part of the
    pending stream per batch. Results stay identical to solo searches."""
    idx, q = index
    rng = np.random.default_rng(4)
    reqs = make_requests(rng, q, 120)
    out = {}
    budget = 24 << 20
    with e8q.Server(idx, mode="precision", max_batch=512, slots=3, memory_budget=budget) as srv:
        def worker(part):
            for j in part:
                qq, k, npb = reqs[j]
                out[j] = srv.submit(qq, k, npb)

        th = [threading.Thread(target=worker, args=(range(t, len(reqs), 4),)) for t in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        res = {j: srv.result(out[j], timeout_ms=60000) for j in range(len(reqs))}
        st = srv.stats(reset=True)
        assert srv.stats()["completed"] == 0  # reset
    assert st["completed"] == len(reqs)
    assert st["peak_batch_bytes"] <= budget
    for j, (qq, k, npb) in enumerate(reqs):
        assert same(res[j], idx.search(qq, k, npb, mode="precision"))


def test_server_errors(e8q, index):
    idx, q = index
    srv = e8q.Server(idx, mode="precision", max_batch=64, max_k=32, max_nprobe=16, memory_budget=64 << 20)
    with pytest.raises(ValueError):
        srv.submit(q[:2], 0, 4)
    with pytest.raises(ValueError):
        srv.submit(q[:2], 33, 4)
    with pytest.raises(ValueError):
        srv.submit(q[:2], 10, 17)
    with pytest.raises(ValueError):
        srv.submit(q[:2, :10], 10, 4)
    with pytest.raises(RuntimeError):
        srv.submit(q[:65], 10, 4)  # larger than a batch: never admissible
    i = srv.submit(q[:3], 10, 4)
    assert srv.result(i, timeout_ms=60000) is not None
    with pytest.raises(IndexError):
        srv.result(i)  # already collected
    assert srv.stats()["rejected"] == 1
    srv.stop()
    with pytest.raises(RuntimeError):
        srv.submit(q[:2], 10, 4)
    with pytest.raises(ValueError):
        e8q.Server(idx, mode="plain")
