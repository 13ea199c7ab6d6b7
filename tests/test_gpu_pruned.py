"""The pruned production search on the GPU (mode "pruned", the default of
E8qIndex.search as in the reference).

Every decision is taken in the reference's order against its running heap
(one warp per query), so it is pinned three ways:
  * against the reference's own pruned search (tests/golden/pruned_*.npz,
    written by the reference compiled from its sources): same top-k ids
    outside ties, distances within 1e-4, and for every query the reference's
    own candidate and survivor counts, on indexes built on the GPU and on the
    reference's own index files;
  * against the oracle's restatement of the same sequential search on other
    inputs (k up to 128, nprobe beyond nlist): survivors per query equal, the
    results agree;
  * with pruning off (set_disable_prune) it is the plain scan.
"""
import glob
import os

import numpy as np
import pytest

from conftest import ROOT, load_golden
from gen import det_mixture
from parity import assert_topk_parity

pytestmark = pytest.mark.gpu

FIXTURES = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "pruned_*.npz")))


@pytest.fixture(scope="module")
def e8q():
    import e8qlib

    return e8qlib


def _case(path):
    g = np.load(path)
    dim, bits, n, nlist, seed, nq, k, nprobe = (int(v) for v in g["params"])
    x, cm, lab = det_mixture(seed, n, dim, nlist, float(g["sigma"]))
    q = det_mixture(seed + 1000, nq, dim, nlist, float(g["sigma"]))[0]
    return g, (dim, bits, n, nlist, seed, nq, k, nprobe), x, cm, lab, q


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[7:-4])
def test_pruned_matches_reference_and_oracle_bound(e8q, oracle_lib, path):
    g, (dim, bits, n, nlist, seed, nq, k, nprobe), x, cm, lab, q = _case(path)
    alpha = float(g["alpha"])
    idx = e8q.E8qIndex(dim, bits, seed)
    idx.build(x, cm, lab, prune_alpha=alpha)
    # the default mode is the reference's pruned search
    ids, d = idx.search(q, k, nprobe)
    assert_topk_parity(ids, d, g["search_ids"], g["search_dists"])
    # query by query and in one batch: the reference's candidates and survivors
    orc = oracle_lib.OracleE8qIndex(x, cm, lab, bits, seed=seed, threads=8)
    assert np.array_equal(orc.banks(), g["banks"])
    surv = np.zeros(nq, np.uint64)
    cand = np.zeros(nq, np.uint64)
    for i in range(nq):
        a, b, st = idx.search(q[i:i + 1], k, nprobe, return_stats=True, mode="pruned")
        assert np.array_equal(a[0], ids[i]) and np.array_equal(b[0], d[i])
        surv[i] = st["survivors"]
        cand[i] = st["candidates"]
    assert np.array_equal(cand, g["candidates"])
    assert np.array_equal(surv, g["survivors"]), (surv, g["survivors"])
    oi, od, oc, osv = orc.search_pruned(q, k, nprobe, alpha=alpha)
    assert np.array_equal(surv, osv)
    assert_topk_parity(ids, d, oi, od)
    # the per-query value kept is the heap's final k-th distance
    thr = idx.pruned_thresholds(1)
    assert thr[0] == d[nq - 1, k - 1]
    # pruning did something at every rate: fewer survivors than candidates
    assert surv.sum() < cand.sum()


def test_pruned_disabled_is_the_plain_scan(e8q):
    g, (dim, bits, n, nlist, seed, nq, k, nprobe), x, cm, lab, q = _case(FIXTURES[0])
    idx = e8q.E8qIndex(dim, bits, seed)
    idx.build(x, cm, lab)
    pi, pd = idx.search(q, k, nprobe, mode="plain")
    idx.set_disable_prune(True)
    ai, ad, st = idx.search(q, k, nprobe, return_stats=True, mode="pruned")
    assert st["survivors"] + min(st["candidates"], nq * max(4 * k, 32)) >= st["candidates"]
    assert_topk_parity(ai, ad, pi, pd)
    # "auto" follows the flag: the plain scan now
    bi, bd = idx.search(q, k, nprobe)
    assert np.array_equal(bi, pi) and np.array_equal(bd, pd)
    assert np.array_equal(idx.pruned_thresholds(nq), ad[:, k - 1])


@pytest.mark.parametrize("name", ["d96_b4", "d100_b1", "d128_b9"])
def test_pruned_on_reference_index_files(e8q, name):
    """An index the reference wrote (its own scan banks, as read from the
    file) searched with the pruned path returns the reference's pruned
    results."""
    path = os.path.join(ROOT, "tests", "golden", f"index_{name}.e8ax")
    g = load_golden(f"pruned_{name}.npz")
    dim, bits, n, nlist, seed, nq, k, nprobe = (int(v) for v in g["params"])
    q = det_mixture(seed + 1000, nq, dim, nlist, float(g["sigma"]))[0]
    idx = e8q.E8qIndex.load(path)
    ids, d = idx.search(q, k, nprobe, mode="pruned")
    assert_topk_parity(ids, d, g["search_ids"], g["search_dists"])


@pytest.mark.parametrize("dim,bits,nlist,nprobe,k", [
    (960, 6, 64, 16, 10), (768, 4, 48, 48, 100), (128, 2, 40, 60, 128), (200, 7, 30, 5, 1)])
def test_pruned_vs_oracle_bound_larger(e8q, oracle_lib, dim, bits, nlist, nprobe, k):
    """Wider lists, k up to 128 and nprobe beyond nlist: the GPU's survivors
    are the oracle's sequential search's, query by query, and so is the top-k
    (ids outside ties, distances within 1e-4)."""
    x, cm, lab = det_mixture(dim * 3 + bits, 12000, dim, nlist, 0.45)
    q = det_mixture(dim * 3 + bits + 9, 12, dim, nlist, 0.45)[0]
    idx = e8q.E8qIndex(dim, bits, 4)
    idx.build(x, cm, lab)
    orc = oracle_lib.OracleE8qIndex(x, cm, lab, bits, seed=4, threads=8)
    surv = np.zeros(len(q), np.uint64)
    ids, d = idx.search(q, k, nprobe, mode="pruned")
    for i in range(len(q)):
        a, b, st = idx.search(q[i:i + 1], k, nprobe, return_stats=True, mode="pruned")
        assert np.array_equal(a[0], ids[i]) and np.array_equal(b[0], d[i])
        surv[i] = st["survivors"]
    oi, od, oc, osv = orc.search_pruned(q, k, nprobe)
    assert np.array_equal(surv, osv)
    assert_topk_parity(ids, d, oi, od)


PROBES = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "probe_bound_*.npz")))


@pytest.mark.parametrize("path", PROBES, ids=lambda p: os.path.basename(p)[12:-4])
def test_probe_bound_w_matches_reference(e8q, oracle_lib, path):
    """E8qIndex.probe_bound_w on the GPU: the reference's values (its
    probe_bound_w on the same build, rates 1, 4 and 9) within 1e-9 relative,
    the oracle's too; NaN for a query index or an id out of range."""
    g = np.load(path)
    dim, bits, n, nlist, seed, nq = (int(v) for v in g["params"])
    x, cm, lab = det_mixture(seed, n, dim, nlist, float(g["sigma"]))
    q = det_mixture(seed + 1000, nq, dim, nlist, float(g["sigma"]))[0]
    idx = e8q.E8qIndex(dim, bits, seed)
    idx.build(x, cm, lab)
    got = idx.probe_bound_w(q, x[g["ids"]], g["qidx"], g["ids"])
    ref = g["out"]
    assert got.dtype == np.float64
    assert np.array_equal(np.isnan(got), np.isnan(ref))
    fin = ~np.isnan(ref)
    assert np.all(np.abs(got[fin] - ref[fin]) <= 1e-9 * np.maximum(np.abs(ref[fin]), 1e-3))
    orc = oracle_lib.OracleE8qIndex(x, cm, lab, bits, seed=seed, threads=8)
    o = orc.probe_bound_w(q, x[g["ids"][:8]], g["qidx"][:8], g["ids"][:8])
    assert np.allclose(got[:8], o, rtol=1e-9, atol=1e-12, equal_nan=True)
    bad = idx.probe_bound_w(q, x[:2], np.array([nq, 0], np.uint32), np.array([0, n + 5], np.uint32))
    assert np.all(np.isnan(bad))
    with pytest.raises(ValueError):
        idx.probe_bound_w(q, x[:3], np.zeros(2, np.uint32), np.zeros(2, np.uint32))
