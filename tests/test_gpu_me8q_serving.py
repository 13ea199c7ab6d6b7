"""ME8Q under captured plans and the serving loop: a ragged batch through a
plan equals the same batch searched directly, and every request served in a
mixed, continuously batched stream equals the same queries searched alone,
bit for bit."""
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
    dim = 320
    x, cm, lab = det_mixture(611, 12000, dim, 40, 0.5)
    idx = e8q.Me8qIndex(dim, 4.0, 3)
    idx.build(x, cm, lab)
    q = det_mixture(612, 500, dim, 40, 0.5)[0]
    return idx, q


def same(a, b):
    return np.array_equal(a[0], b[0]) and np.array_equal(a[1].view(np.uint32), b[1].view(np.uint32))


def test_me8q_search_ragged_matches_uniform(e8q, index):
    idx, q = index
    rng = np.random.default_rng(1)
    k = rng.integers(1, 65, len(q)).astype(np.uint32)
    npb = rng.integers(1, 41, len(q)).astype(np.uint32)
    ids, d = idx.search_ragged(q, k, npb, 64)
    for i in range(0, len(q), 37):
        ai, ad = idx.search(q[i:i + 1], int(k[i]), int(npb[i]), mode="batched")
        assert np.array_equal(ids[i, :k[i]], ai[0]) and np.array_equal(d[i, :k[i]].view(np.uint32),
                                                                       ad[0].view(np.uint32)), i
        assert np.all(ids[i, k[i]:] == 0xFFFFFFFF) and np.all(np.isinf(d[i, k[i]:]))


def test_me8q_plan_matches_direct(e8q, index):
    idx, q = index
    rng = np.random.default_rng(2)
    plan = e8q.Plan(idx, max_queries=300, k_max=32, nprobe_max=24)
    for nq in (1, 64, 65, 300):
        qq = q[:nq]
        k = rng.integers(1, 33, nq).astype(np.uint32)
        npb = rng.integers(1, 25, nq).astype(np.uint32)
        got = plan.run(qq, k, npb)
        ref = idx.search_ragged(qq, k, npb, 32)
        assert same(got, ref), nq
    with pytest.raises(ValueError):
        e8q.Plan(idx, mode="plain", max_queries=64)


@pytest.mark.parametrize("mode", ["batched", "precision"])
def test_me8q_server_matches_alone(e8q, index, mode):
    idx, q = index
    rng = np.random.default_rng(3)
    reqs, off = [], 0
    for _ in range(70):
        m = int(rng.integers(1, 17))
        if off + m > len(q):
            off = 0
        reqs.append((q[off:off + m], int(rng.choice([1, 10, 100])), int(rng.integers(1, 41))))
        off += m
    with e8q.Server(idx, mode=mode, max_batch=256, slots=2) as srv:
        ids = [srv.submit(qq, k, npb) for qq, k, npb in reqs]
        got = [srv.result(i, timeout_ms=60000) for i in ids]
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert 0 < st["p50_ms"] <= st["p99_ms"]
    for (qq, k, npb), res in zip(reqs, got):
        assert res is not None
        assert same(res, idx.search(qq, k, npb, mode=mode)), (k, npb)


def test_me8q_precision_plan_matches_direct(e8q, index):
    idx, q = index
    rng = np.random.default_rng(5)
    plan = e8q.Plan(idx, mode="precision", max_queries=200, k_max=16, nprobe_max=24)
    for nq in (3, 64, 200):
        qq = q[:nq]
        k = rng.integers(1, 17, nq).astype(np.uint32)
        npb = rng.integers(1, 25, nq).astype(np.uint32)
        assert same(plan.run(qq, k, npb), idx.search_ragged(qq, k, npb, 16, mode="precision")), nq
