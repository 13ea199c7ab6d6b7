"""Me8qIndex.search's default mode: the reference's production FastScan
cascade (me8q_fast.cpp SearchIVFFast*) on the GPU, against

  * the reference's own outputs (tests/golden/me8q_pruned_*.npz: rows,
    distances and per-query candidate / survivor counts),
  * the oracle's restatement (orc_me8q_search_pruned) on other inputs,
    multi-run plans, k up to 128 and batches.

Every prune decision is taken in the reference's order against the same
running heap, so the rows are the reference's; a row may differ only where
a run score summed in another order moves a distance across a decision by
its last bits (the tests allow 5 % of rows), and the distances of equal rows
agree within 1e-5 relative."""
import numpy as np
import pytest

from conftest import load_golden
from gen import det_mixture
from parity import assert_topk_parity, rel_err

pytestmark = pytest.mark.gpu

CASES = ["d200_a4", "d200_spec", "d96_a6_k20", "d150_a3_a001", "d64_a1"]


@pytest.fixture(scope="module")
def e8q():
    import e8qlib

    return e8qlib


def _same_rows(a, b):
    return np.array([np.array_equal(x, y) for x, y in zip(a, b)])


def _dist_agree(ids, d, ref_ids, ref_d, same):
    if same.any():
        assert rel_err(d[same], ref_d[same]).max() < 1e-5


@pytest.mark.parametrize("name", CASES)
def test_pruned_matches_reference(e8q, name):
    G = load_golden(f"me8q_pruned_{name}.npz")
    dim, seed, n, nlist, nq, k, nprobe = (int(v) for v in G["params"])
    avg, sigma, spec, alpha = float(G["avg_bits"]), float(G["sigma"]), str(G["plan_spec"]), float(G["alpha"])
    x, cm, lab = det_mixture(seed + 5000 + dim, n, dim, nlist, sigma)
    q = det_mixture(seed + 6000 + dim, nq, dim, nlist, sigma)[0]
    m = e8q.Me8qIndex(dim, avg, seed)
    m.build(x, cm, lab, plan_spec=spec, prune_alpha=alpha)
    ids, d, st = m.search(q, k, nprobe, return_stats=True)
    same = _same_rows(ids, G["search_ids"])
    assert same.mean() >= 0.95, same.mean()
    _dist_agree(ids, d, G["search_ids"], G["search_dists"], same)
    # every probed row is a candidate; the survivors are the reference's
    assert st["candidates"] == int(G["candidates"].sum())
    assert abs(st["survivors"] - int(G["survivors"].sum())) <= 0.02 * int(G["survivors"].sum()) + 2
    # one query at a time: the same rows (queries are independent)
    for i in range(0, nq, 7):
        a, b = m.search(q[i:i + 1], k, nprobe)
        assert np.array_equal(a[0], ids[i]) and np.array_equal(b[0], d[i])


@pytest.mark.parametrize("dim,avg,k,nprobe,alpha,spec", [
    (256, 3.0, 10, 6, 0.0, "64:5,64:3,64:2,64:0"),  # three coded runs and a dropped one
    (192, 4.0, 50, 5, 0.3, "64:6,64:4,64:1"),       # a rate-1 run
    (128, 2.0, 128, 8, 0.0, "64:3,64:1"),
    (256, 3.0, 10, 6, 0.0, ""),                     # the DP plan of a power-law spectrum: 64:8, 192:1
])
def test_pruned_matches_oracle(e8q, oracle_lib, dim, avg, k, nprobe, alpha, spec):
    nlist = 12
    x, cm, lab = det_mixture(700 + dim, 5000, dim, nlist, 0.5)
    q = det_mixture(800 + dim, 48, dim, nlist, 0.5)[0]
    var = ((np.arange(dim) + 1.0) ** -1.5).astype(np.float32)
    m = e8q.Me8qIndex(dim, avg, 5)
    m.build(x, cm, lab, variance=var, prune_alpha=alpha, plan_spec=spec)
    orc = oracle_lib.OracleMe8qIndex(x, cm, lab, avg_bits=avg, seed=5, variance=var, plan_spec=spec, threads=4)
    assert [list(p) for p in m.plan] == [list(p) for p in orc.plan]
    assert sum(1 for p in orc.plan if p[1]) >= 2  # a multi-run plan
    ids, d, st = m.search(q, k, nprobe, return_stats=True)
    oi, od, oc, os_ = orc.search_pruned(q, k, nprobe, alpha=alpha, threads=4)
    same = _same_rows(ids, oi)
    assert same.mean() >= 0.95, same.mean()
    _dist_agree(ids, d, oi, od, same)
    assert st["candidates"] == int(oc.sum())
    assert abs(st["survivors"] - int(os_.sum())) <= 0.02 * int(os_.sum()) + 2
    # the cascade prunes; with a tiny alpha it returns the exact scan's rows
    assert st["survivors"] < st["candidates"]
    m2 = e8q.Me8qIndex(dim, avg, 5)
    m2.build(x, cm, lab, variance=var, prune_alpha=1e-9, plan_spec=spec)
    a, b = m2.search(q, k, nprobe)
    e, f = m2.search(q, k, nprobe, mode="batched")
    assert_topk_parity(a, b, e, f)


def test_pruned_edges(e8q, oracle_lib):
    dim, nlist = 96, 6
    x, cm, lab = det_mixture(901, 700, dim, nlist, 0.5)
    q = det_mixture(902, 9, dim, nlist, 0.5)[0]
    m = e8q.Me8qIndex(dim, 4.0, 1)
    m.build(x, cm, lab)
    orc = oracle_lib.OracleMe8qIndex(x, cm, lab, avg_bits=4.0, seed=1, threads=4)
    # nprobe above the list count, k above what the probed lists hold
    for k, nprobe in ((10, 50), (128, 2), (1, 1)):
        ids, d = m.search(q, k, nprobe)
        oi, od, _, _ = orc.search_pruned(q, k, nprobe, threads=4)
        assert _same_rows(ids, oi).mean() >= 0.9
        pad = ids == np.uint32(0xFFFFFFFF)
        assert np.array_equal(pad, oi == np.uint32(0xFFFFFFFF))
        assert np.all(np.isinf(d[pad]))
    # an empty batch, and the other modes still reachable
    e_ids, _ = m.search(np.zeros((0, dim), np.float32), 10, 4)
    assert e_ids.shape == (0, 10)
    with pytest.raises(ValueError):
        m.search(q, 10, 4, mode="plain")
