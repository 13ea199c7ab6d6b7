"""The oracle's restatement of the reference's production (pruned) search,
pinned to the reference's own results (tests/golden/pruned_*.npz, written by
tests/golden/make_golden.py from the reference compiled from its sources):
scan-bank headers byte for byte, and per query the same ids, the same number
of scanned candidates and the same number of survivors refined exactly, at
rates 1, 2, 4, 5, 6 and 9 and two prune budgets. Distances agree within 1e-6
relative (the reference's AVX-512 routing GEMV accumulates d2 in fp32, the
oracle in fp64 like the reference's scalar kernel)."""
import glob
import os

import numpy as np
import pytest

from conftest import ROOT
from gen import det_mixture

FIXTURES = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "pruned_*.npz")))


def test_fixtures_present():
    assert len(FIXTURES) >= 6


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[7:-4])
def test_oracle_pruned_search_matches_reference(oracle_lib, path):
    O = oracle_lib
    g = np.load(path)
    dim, bits, n, nlist, seed, nq, k, nprobe = (int(v) for v in g["params"])
    x, cm, lab = det_mixture(seed, n, dim, nlist, float(g["sigma"]))
    q = det_mixture(seed + 1000, nq, dim, nlist, float(g["sigma"]))[0]
    orc = O.OracleE8qIndex(x, cm, lab, bits, seed=seed, threads=8)
    assert np.array_equal(orc.banks(), g["banks"]), "scan-bank headers differ from the reference's"
    ids, dists, cand, surv = orc.search_pruned(q, k, nprobe, alpha=float(g["alpha"]))
    assert np.array_equal(ids, g["search_ids"])
    ref_d = g["search_dists"]
    fin = np.isfinite(ref_d)
    assert np.array_equal(np.isfinite(dists), fin)
    rel = np.abs(dists[fin].astype(np.float64) - ref_d[fin]) / np.maximum(np.abs(ref_d[fin]), 1e-3)
    assert rel.max() < 1e-6
    assert np.array_equal(cand, g["candidates"])
    assert np.array_equal(surv, g["survivors"])
    # pruning did work: fewer survivors than candidates, and the plain scan
    # (pruning off) refines every candidate and finds the same top-k here
    assert surv.sum() < cand.sum()
    pid, pdist, pc, ps = orc.search_pruned(q, k, nprobe, alpha=float(g["alpha"]), disable_prune=True)
    assert np.array_equal(ps, pc)


def test_ortho_quantile_values(oracle_lib):
    O = oracle_lib
    L = O.lib()
    # lambda = PhiInv(1 - alpha / k_eff), floored at 1
    assert abs(L.orc_phi_inv(0.975) - 1.959963984540054) < 1e-12
    assert abs(L.orc_ortho_quantile(1.0, 40) - 1.959964) < 1e-6
    assert L.orc_ortho_quantile(1.0, 1) == 1.0  # tail capped at 0.49 -> PhiInv(0.51) < 1


PROBES = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "probe_bound_*.npz")))


@pytest.mark.parametrize("path", PROBES, ids=lambda p: os.path.basename(p)[12:-4])
def test_oracle_probe_bound_w_matches_reference(oracle_lib, path):
    """ProbeBoundW: the bound's normalised discrepancy per (query, stored
    vector) pair, every term in double; the reference's values (its
    probe_bound_w, at rates 1, 4 and 9) within 1e-9 relative."""
    g = np.load(path)
    dim, bits, n, nlist, seed, nq = (int(v) for v in g["params"])
    x, cm, lab = det_mixture(seed, n, dim, nlist, float(g["sigma"]))
    q = det_mixture(seed + 1000, nq, dim, nlist, float(g["sigma"]))[0]
    orc = oracle_lib.OracleE8qIndex(x, cm, lab, bits, seed=seed, threads=8)
    got = orc.probe_bound_w(q, x[g["ids"]], g["qidx"], g["ids"])
    ref = g["out"]
    assert np.array_equal(np.isnan(got), np.isnan(ref))
    fin = ~np.isnan(ref)
    assert np.all(np.abs(got[fin] - ref[fin]) <= 1e-9 * np.maximum(np.abs(ref[fin]), 1e-3))
