"""Autotuning and captured (CUDA graph) plans on the GPU: a plan's results are
bitwise those of the eager ragged search for every batch size, including
sizes between captured buckets and repeated runs; autotuning picks a valid
setting and never changes results."""
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
    dim, bits = 256, 5
    x, cm, lab = det_mixture(601, 9000, dim, 40, 0.5)
    idx = e8q.E8qIndex(dim, bits, 11)
    idx.build(x, cm, lab)
    q = det_mixture(602, 300, dim, 40, 0.5)[0]
    return idx, q


def same(a, b):
    return np.array_equal(a[0], b[0]) and np.array_equal(a[1].view(np.uint32), b[1].view(np.uint32))


@pytest.mark.parametrize("mode", ["precision", "batched"])
def test_plan_matches_eager(e8q, index, mode):
    idx, q = index
    rng = np.random.default_rng(5)
    plan = e8q.Plan(idx, mode=mode, max_queries=200, k_max=16, nprobe_max=24, autotune=(mode == "precision"))
    for nq in (1, 63, 64, 65, 130, 200, 64):
        qq = q[:nq]
        ks = rng.integers(1, 17, nq).astype(np.uint32)
        nps = rng.integers(1, 25, nq).astype(np.uint32)
        got = plan.run(qq, ks, nps)
        ref = idx.search_ragged(qq, ks, nps, 16, mode=mode)
        assert same(got, ref), nq
    # scalar k / nprobe
    got = plan.run(q[:10], 10, 8)
    ref = idx.search(q[:10], 10, 8, mode=mode)
    assert np.array_equal(got[0][:, :10], ref[0]) and np.array_equal(got[1][:, :10], ref[1])
    with pytest.raises(ValueError):
        plan.run(q[:201], 10, 8)
    with pytest.raises(ValueError):
        plan.run(q[:2], 17, 8)
    with pytest.raises(ValueError):
        plan.run(q[:2], 10, 25)


def test_autotune_keeps_results(e8q, index):
    idx, q = index
    before = idx.search(q[:150], 10, 12, mode="precision")
    t = idx.autotune("precision", 150, 10, 12)
    assert t["schedule"] in ("longest_list_first", "list_id_order")
    assert t["stages"] in (4, 6, 8)
    assert 0 < t["best_ms"] <= t["default_ms"]
    after = idx.search(q[:150], 10, 12, mode="precision")
    assert same(before, after)
    tb = idx.autotune("batched", 150, 10, 12)
    assert tb["stages"] == 6 and tb["best_ms"] > 0
    assert same(idx.search(q[:150], 10, 12, mode="batched"), idx.search(q[:150], 10, 12, mode="batched"))
    with pytest.raises(ValueError):
        idx.autotune("plain", 10, 10, 4)


def test_search_replays_graph_of_repeated_shape(e8q):
    """search() calls of a repeated shape (1,024+ queries, grouped modes)
    replay a captured graph: the results equal the direct path's (a ragged
    call with the same uniform k / nprobe), for new query contents, and after
    a rebuild of the index."""
    from gen import det_mixture

    dim, nlist = 128, 24
    x, cm, lab = det_mixture(61, 3000, dim, nlist, 0.5)
    idx = e8q.E8qIndex(dim, 5, 1)
    idx.build(x, cm, lab)
    n = 1100
    ks = np.full(n, 10, np.uint32)
    nps = np.full(n, 6, np.uint32)
    for mode in ("precision", "batched"):
        for seed in (62, 63, 64, 65):  # direct, capture, replay, replay
            q = det_mixture(seed, n, dim, nlist, 0.5)[0]
            ids, d = idx.search(q, 10, 6, mode=mode)
            rids, rd = idx.search_ragged(q, ks, nps, 10, mode=mode)
            assert np.array_equal(ids, rids) and np.array_equal(d.view(np.uint32), rd.view(np.uint32)), (mode, seed)
    x2, cm2, lab2 = det_mixture(66, 3000, dim, nlist, 0.5)
    idx.build(x2, cm2, lab2)
    for seed in (67, 68, 69):
        q = det_mixture(seed, n, dim, nlist, 0.5)[0]
        ids, d = idx.search(q, 10, 6, mode="batched")
        rids, rd = idx.search_ragged(q, ks, nps, 10, mode="batched")
        assert np.array_equal(ids, rids) and np.array_equal(d.view(np.uint32), rd.view(np.uint32)), seed
