"""The pruned production search on the GPU (mode "pruned", the default of
E8qIndex.search as in the reference).

Pinned three ways:
  * against the reference's own pruned search (tests/golden/pruned_*.npz,
    written by the reference compiled from its sources): same top-k ids
    outside ties, distances within 1e-4, on indexes built on the GPU and on
    the reference's own index files;
  * against the oracle's restatement of the same bound with the GPU's
    per-query threshold: for every query the number of vectors that survive
    the bound and are refined is exactly the oracle's (the LUT, the banks and
    every fused operation of the bound are the reference's bit for bit), and
    the results agree;
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
    # query by query: the survivors of the bound at the GPU's threshold are
    # exactly the oracle's
    orc = oracle_lib.OracleE8qIndex(x, cm, lab, bits, seed=seed, threads=8)
    assert np.array_equal(orc.banks(), g["banks"])
    thr = np.zeros(nq, np.float32)
    surv = np.zeros(nq, np.uint64)
    cand = np.zeros(nq, np.uint64)
    for i in range(nq):
        a, b, st = idx.search(q[i:i + 1], k, nprobe, return_stats=True, mode="pruned")
        assert_topk_parity(a, b, g["search_ids"][i:i + 1], g["search_dists"][i:i + 1])
        thr[i] = idx.pruned_thresholds(1)[0]
        surv[i] = st["survivors"]
        cand[i] = st["candidates"]
    oi, od, oc, osv = orc.search_pruned_at(q, k, nprobe, thr=thr, alpha=alpha)
    assert np.array_equal(cand, oc)
    assert np.array_equal(surv, osv), (surv, osv)
    assert_topk_parity(ids, d, oi, od)
    # the threshold is an upper bound of the answer's k-th distance
    kth = g["search_dists"][:, -1].astype(np.float64)
    fin = np.isfinite(kth)
    assert np.all(thr[fin] >= kth[fin] - 1e-4 * np.abs(kth[fin]))
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
    assert np.all(np.isinf(idx.pruned_thresholds(nq)))


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
    """Wider lists, k up to 128 and nprobe beyond nlist: the GPU's survivors at
    its threshold are the oracle's, and the top-k is the plain scan's outside
    ties wherever the bound held (checked against the oracle's result at the
    same threshold)."""
    x, cm, lab = det_mixture(dim * 3 + bits, 12000, dim, nlist, 0.45)
    q = det_mixture(dim * 3 + bits + 9, 12, dim, nlist, 0.45)[0]
    idx = e8q.E8qIndex(dim, bits, 4)
    idx.build(x, cm, lab)
    orc = oracle_lib.OracleE8qIndex(x, cm, lab, bits, seed=4, threads=8)
    thr = np.zeros(len(q), np.float32)
    surv = np.zeros(len(q), np.uint64)
    ids = np.zeros((len(q), k), np.uint32)
    d = np.zeros((len(q), k), np.float32)
    for i in range(len(q)):
        a, b, st = idx.search(q[i:i + 1], k, nprobe, return_stats=True, mode="pruned")
        ids[i], d[i] = a[0], b[0]
        thr[i] = idx.pruned_thresholds(1)[0]
        surv[i] = st["survivors"]
    oi, od, oc, osv = orc.search_pruned_at(q, k, nprobe, thr=thr)
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
