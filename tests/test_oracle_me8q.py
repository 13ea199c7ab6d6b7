"""The ME8Q restatement (oracle/me8q_oracle.c) against fixtures produced by
the reference's own Me8qIndex (tests/golden/make_golden.py): the DP plan, the
cluster-major ids, every segment code (digits, branch), the per-segment
(coef, h2) factors, estimates and the plain search."""
import numpy as np
import pytest

from conftest import load_golden
from gen import det_mixture
from parity import assert_topk_parity, rel_err

CASES = ["me8q_d200_spec", "me8q_d200_a4", "me8q_d150_a3", "me8q_d96_a6"]


@pytest.mark.parametrize("name", CASES)
def test_me8q_oracle_matches_reference(oracle_lib, name):
    G = load_golden(name + ".npz")
    dim, seed, n, nlist, nq, k, nprobe = (int(v) for v in G["params"])
    avg, sigma, spec = float(G["avg_bits"]), float(G["sigma"]), str(G["plan_spec"])
    x, cm, lab = det_mixture(seed + 5000 + dim, n, dim, nlist, sigma)
    q = det_mixture(seed + 6000 + dim, nq, dim, nlist, sigma)[0]
    orc = oracle_lib.OracleMe8qIndex(x, cm, lab, avg_bits=avg, seed=seed, plan_spec=spec, threads=4)
    assert [list(p) for p in G["plan"]] == [list(p) for p in orc.plan]
    assert np.array_equal(orc.ids, G["ids"])
    for pos in range(n):
        dg, br, cf, h2 = orc.codes(pos)
        assert np.array_equal(dg, G["digits"][pos]), pos
        assert np.array_equal(br, G["branch"][pos]), pos
        assert np.array_equal(cf.view(np.uint32), G["coef"][pos].view(np.uint32)), pos
        assert np.array_equal(h2.view(np.uint32), G["h2"][pos].view(np.uint32)), pos
    est = np.array([[orc.estimate(q[i], int(g)) for g in G["est_ids"]] for i in range(nq)], np.float32)
    assert rel_err(est, G["est"]).max() < 1e-6
    ids, d = orc.search(q, k, nprobe)
    assert_topk_parity(ids, d, G["search_ids"], G["search_dists"], rtol=1e-6)


def test_me8q_plan_edges(oracle_lib):
    O = oracle_lib
    # flat variance: one uniform run at the average rate
    assert O.me8q_allocate(np.ones(256, np.float32), 4.0) == [(256, 4)]
    # dead tail dims are dropped; the cap (nblocks/2 runs) holds
    var = np.concatenate([np.linspace(4, 1, 192), np.zeros(64)]).astype(np.float32)
    plan = O.me8q_allocate(var, 3.0)
    assert sum(p[0] for p in plan) == 256 and plan[-1][1] == 0 and len(plan) <= 2
    assert O.parse_plan_spec("64:3,64:0", 128) == [(64, 3), (64, 0)]
    with pytest.raises(ValueError):
        O.parse_plan_spec("64:3", 128)
    with pytest.raises(ValueError):
        O.parse_plan_spec("60:3,68:0", 128)


PRUNED_CASES = ["d200_a4", "d200_spec", "d96_a6_k20", "d150_a3_a001", "d64_a1",
                "d192_k100_np_all", "d256_spec_r1"]


@pytest.mark.parametrize("name", PRUNED_CASES)
def test_me8q_pruned_oracle_matches_reference(oracle_lib, name):
    """The restated FastScan cascade (orc_me8q_search_pruned) against the
    reference's own Me8qIndex.search: every row, its distances, and each
    query's scanned candidates and survivors."""
    G = load_golden(f"me8q_pruned_{name}.npz")
    dim, seed, n, nlist, nq, k, nprobe = (int(v) for v in G["params"])
    avg, sigma, spec, alpha = float(G["avg_bits"]), float(G["sigma"]), str(G["plan_spec"]), float(G["alpha"])
    x, cm, lab = det_mixture(seed + 5000 + dim, n, dim, nlist, sigma)
    q = det_mixture(seed + 6000 + dim, nq, dim, nlist, sigma)[0]
    orc = oracle_lib.OracleMe8qIndex(x, cm, lab, avg_bits=avg, seed=seed, plan_spec=spec, threads=4)
    ids, d, cand, surv = orc.search_pruned(q, k, nprobe, alpha=alpha, threads=4)
    assert np.array_equal(ids, G["search_ids"])
    assert rel_err(d, G["search_dists"]).max() < 1e-6
    assert np.array_equal(cand, G["candidates"]) and np.array_equal(surv, G["survivors"])
    # the cascade prunes: most scanned rows never reach the heap
    assert surv.sum() < 0.2 * cand.sum()
