"""GPU batched path (persistent work-queue kernel) against the oracle, the
plain path, and itself under different batch compositions."""
import numpy as np
import pytest

from gen import det_mixture, det_normal
from parity import assert_topk_parity

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def e8q():
    import e8qlib

    return e8qlib


@pytest.mark.parametrize("dim,bits,nlist,nprobe,k,nq", [
    (128, 4, 32, 8, 10, 300), (960, 6, 16, 4, 10, 70), (768, 5, 24, 24, 100, 40),
    (200, 3, 20, 7, 32, 130), (64, 13, 8, 3, 128, 20), (128, 1, 12, 5, 7, 65), (320, 8, 10, 2, 50, 33)])
def test_batched_vs_oracle(e8q, oracle_lib, dim, bits, nlist, nprobe, k, nq):
    x, cm, lab = det_mixture(dim * 3 + bits, 2500, dim, nlist, 0.5)
    q = det_mixture(dim * 3 + bits + 11, nq, dim, nlist, 0.5)[0]
    idx = e8q.E8qIndex(dim, bits, 9)
    idx.build(x, cm, lab)
    orc = oracle_lib.OracleE8qIndex(x, cm, lab, bits, seed=9, threads=4)
    ids, d = idx.search(q, k, nprobe, mode="batched")
    rids, rd = orc.search(q, k, nprobe, threads=4)
    assert_topk_parity(ids, d, rids, rd)
    pids, pdist = idx.search(q, k, nprobe, mode="plain")
    assert_topk_parity(ids, d, pids, pdist)


def test_batched_alone_equals_in_mix(e8q):
    """Serving invariant: a query's result is the same (bitwise) alone and
    inside any batch, with any neighbours' k and nprobe."""
    dim, bits = 256, 5
    x, cm, lab = det_mixture(31, 6000, dim, 40, 0.5)
    q = det_mixture(32, 200, dim, 40, 0.5)[0]
    idx = e8q.E8qIndex(dim, bits, 2)
    idx.build(x, cm, lab)
    rng = np.random.default_rng(0)
    ks = rng.integers(1, 65, 200).astype(np.uint32)
    nps = rng.integers(1, 41, 200).astype(np.uint32)
    ids, d = idx.search_ragged(q, ks, nps, 64)
    for i in rng.choice(200, 12, replace=False):
        a_ids, a_d = idx.search_ragged(q[i:i + 1], ks[i:i + 1], nps[i:i + 1], 64)
        assert np.array_equal(a_ids[0], ids[i]) and np.array_equal(a_d[0].view(np.uint32), d[i].view(np.uint32))
        # uniform call with the same k / nprobe gives the same list
        u_ids, u_d = idx.search(q[i:i + 1], int(ks[i]), int(nps[i]), mode="batched")
        assert np.array_equal(u_ids[0], ids[i][:ks[i]])
        assert np.array_equal(u_d[0].view(np.uint32), d[i][:ks[i]].view(np.uint32))
        assert np.all(ids[i][ks[i]:] == 0xFFFFFFFF) and np.all(np.isinf(d[i][ks[i]:]))
    # a different mix around the same queries
    perm = rng.permutation(200)
    ids2, d2 = idx.search_ragged(q[perm], ks[perm], nps[perm], 64)
    assert np.array_equal(ids2, ids[perm]) and np.array_equal(d2.view(np.uint32), d[perm].view(np.uint32))


def test_ragged_vs_oracle(e8q, oracle_lib):
    dim, bits = 128, 6
    x, cm, lab = det_mixture(41, 3000, dim, 30, 0.5)
    q = det_normal(42, (50, dim))
    idx = e8q.E8qIndex(dim, bits, 4)
    idx.build(x, cm, lab)
    orc = oracle_lib.OracleE8qIndex(x, cm, lab, bits, seed=4)
    ks = np.array([1, 5, 10, 32, 100, 128] * 9, np.uint32)[:50]
    nps = np.array([1, 2, 3, 30, 100, 7, 16] * 8, np.uint32)[:50]
    ids, d = idx.search_ragged(q, ks, nps, 128)
    for i in range(50):
        rids, rd = orc.search(q[i:i + 1], int(ks[i]), int(nps[i]))
        assert_topk_parity(ids[i:i + 1, :ks[i]], d[i:i + 1, :ks[i]], rids, rd)
    with pytest.raises(ValueError):
        idx.search_ragged(q[:2], np.array([0, 1], np.uint32), np.array([1, 1], np.uint32), 8)
    with pytest.raises(ValueError):
        idx.search_ragged(q[:2], np.array([9, 1], np.uint32), np.array([1, 1], np.uint32), 8)
