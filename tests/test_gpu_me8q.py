"""GPU parity of the ME8Q (mixed-rate) index against the reference's fixtures
and the oracle: the plan, ids, every segment code, the (coef, h2) factors
bit for bit; estimates and search results within fp32 rounding. Everything
runs the CUDA library through e8qlib.Me8qIndex (the C ABI)."""
import numpy as np
import pytest

from conftest import load_golden
from gen import det_mixture
from parity import assert_topk_parity, rel_err

pytestmark = pytest.mark.gpu

GOLDEN = ["me8q_d200_spec", "me8q_d200_a4", "me8q_d150_a3", "me8q_d96_a6"]
# The scan folds each run's coef into its decoded levels and sums in fp32;
# the reference sums per-run fp32 scores in fp64.
RTOL = 1e-4


@pytest.fixture(scope="module")
def e8q():
    import e8qlib

    return e8qlib


def _assert_codes_equal(idx, ids, dg, br, cf, h2):
    gi, gd, gb, gc, gh = idx.export_codes()
    assert np.array_equal(gi, ids)
    bad = np.nonzero((gd != dg).any(axis=1))[0]
    assert bad.size == 0, f"digits differ at rows {bad[:10]}"
    assert np.array_equal(gb, br)
    assert np.array_equal(gc.view(np.uint32), np.asarray(cf, np.float32).view(np.uint32))
    assert np.array_equal(gh.view(np.uint32), np.asarray(h2, np.float32).view(np.uint32))


@pytest.mark.parametrize("name", GOLDEN)
def test_me8q_gpu_matches_reference_fixtures(e8q, name):
    G = load_golden(name + ".npz")
    dim, seed, n, nlist, nq, k, nprobe = (int(v) for v in G["params"])
    avg, sigma, spec = float(G["avg_bits"]), float(G["sigma"]), str(G["plan_spec"])
    x, cm, lab = det_mixture(seed + 5000 + dim, n, dim, nlist, sigma)
    q = det_mixture(seed + 6000 + dim, nq, dim, nlist, sigma)[0]
    idx = e8q.Me8qIndex(dim, avg, seed)
    idx.build(x, cm, lab, plan_spec=spec)
    assert idx.is_built and idx.n == n and idx.num_clusters == nlist
    assert [list(p) for p in idx.plan] == [list(p) for p in G["plan"]]
    ncoded = sum(1 for p in idx.plan if p[1])
    bpv = ncoded * 8 + sum(p[0] // 8 * p[1] for p in idx.plan)
    assert idx.bits_per_dim == pytest.approx(8.0 * bpv / dim)
    _assert_codes_equal(idx, G["ids"], G["digits"], G["branch"], G["coef"], G["h2"])
    est = np.array([[idx.estimate(q[i], int(g)) for g in G["est_ids"]] for i in range(nq)], np.float32)
    assert rel_err(est, G["est"]).max() < 1e-6
    ids, d = idx.search(q, k, nprobe, mode="batched")
    assert_topk_parity(ids, d, G["search_ids"], G["search_dists"], rtol=RTOL)


def _build_both(e8q, oracle_lib, x, cm, lab, **kw):
    okw = {k2: v for k2, v in kw.items() if k2 in ("avg_bits", "seed", "variance", "drop_energy", "plan_spec",
                                                      "extra_budget_bits")}
    orc = oracle_lib.OracleMe8qIndex(x, cm, lab, threads=8, **okw)
    idx = e8q.Me8qIndex(x.shape[1], kw.get("avg_bits", 4.0), kw.get("seed", 0))
    bkw = {k2: v for k2, v in kw.items() if k2 in ("variance", "drop_energy", "plan_spec", "extra_budget_bits")}
    idx.build(x, cm, lab, **bkw)
    return orc, idx


def _oracle_codes(orc):
    rows = [orc.codes(p) for p in range(orc.n)]
    return (np.stack([r[0] for r in rows]), np.stack([r[1] for r in rows]),
            np.stack([r[2] for r in rows]), np.stack([r[3] for r in rows]))


@pytest.mark.parametrize("dim,avg,seed,kw", [
    (768, 3.0, 0, {}),
    (960, 4.0, 21, {}),
    (300, 2.0, 5, {"extra_budget_bits": 40.0}),
    (250, 4.0, 3, {"plan_spec": "64:3,64:0,128:5", "drop_energy": False}),
    (130, 1.0, 8, {}),
])
def test_me8q_gpu_matches_oracle(e8q, oracle_lib, dim, avg, seed, kw):
    n, nlist, nq = 6000, 24, 48
    x, cm, lab = det_mixture(9000 + dim + seed, n, dim, nlist, 0.6)
    q = det_mixture(9100 + dim + seed, nq, dim, nlist, 0.6)[0]
    orc, idx = _build_both(e8q, oracle_lib, x, cm, lab, avg_bits=avg, seed=seed, **kw)
    assert [tuple(p) for p in idx.plan] == [tuple(p) for p in orc.plan]
    _assert_codes_equal(idx, orc.ids, *_oracle_codes(orc))
    for gid in (0, 17, n // 2, n - 1):
        a, b = idx.estimate(q[0], gid), orc.estimate(q[0], gid)
        assert rel_err(a, b) < 1e-6, gid
    for k, nprobe in ((10, 4), (64, 24), (128, 2)):
        ids, d = idx.search(q, k, nprobe, mode="batched")
        oi, od = orc.search(q, k, nprobe)
        assert_topk_parity(ids, d, oi, od, rtol=RTOL)


def test_me8q_gpu_given_variance_and_ragged_lists(e8q, oracle_lib):
    """A caller's variance; lists of every size including empty ones and
    lists shorter than a 32-vector tile; k beyond the probed vectors pads
    with UINT32_MAX / +inf; nprobe beyond nlist is clamped."""
    rng = np.random.default_rng(12)
    dim, nlist = 200, 40
    sizes = np.array([0, 1, 31, 32, 33, 0, 5, 64, 97, 2] * 4)
    lab = np.repeat(np.arange(nlist, dtype=np.uint32), sizes)
    rng.shuffle(lab)
    cm = rng.standard_normal((nlist, dim)).astype(np.float32) * 3
    x = (cm[lab] + rng.standard_normal((lab.size, dim)).astype(np.float32)).astype(np.float32)
    var = np.linspace(2.0, 0.01, dim).astype(np.float32)
    q = (cm[rng.integers(0, nlist, 20)] + rng.standard_normal((20, dim))).astype(np.float32)
    orc, idx = _build_both(e8q, oracle_lib, x, cm, lab, avg_bits=3.0, seed=4, variance=var)
    assert [tuple(p) for p in idx.plan] == [tuple(p) for p in orc.plan]
    _assert_codes_equal(idx, orc.ids, *_oracle_codes(orc))
    for k, nprobe in ((10, 3), (128, 2), (5, 1000)):
        ids, d = idx.search(q, k, nprobe, mode="batched")
        oi, od = orc.search(q, k, nprobe)
        assert_topk_parity(ids, d, oi, od, rtol=RTOL)
    empty_ids, empty_d = idx.search(np.zeros((0, dim), np.float32), 10, 4)
    assert empty_ids.shape == (0, 10) and empty_d.shape == (0, 10)
    with pytest.raises(IndexError):
        idx.estimate(q[0], lab.size + 5)
    with pytest.raises(ValueError):
        idx.search(q, 0, 4)
    with pytest.raises(ValueError):
        idx.search(q, 10, 0)
    with pytest.raises(ValueError):
        idx.search(q[:, :10], 10, 4)


def test_me8q_gpu_rebuild_is_deterministic(e8q):
    x, cm, lab = det_mixture(4242, 3000, 384, 16, 0.5)
    a = e8q.Me8qIndex(384, 3.5, 77)
    a.build(x, cm, lab)
    first = a.export_codes()
    a.build(x, cm, lab)
    second = a.export_codes()
    for u, v in zip(first, second):
        assert np.array_equal(np.asarray(u).view(np.uint8), np.asarray(v).view(np.uint8))
    assert a.memory_bytes > 0


def test_me8q_gpu_all_dropped_plan(e8q, oracle_lib):
    """A plan with no coded run: every estimate is the routing distance plus
    nothing, identical to the oracle's."""
    x, cm, lab = det_mixture(777, 500, 128, 6, 0.5)
    q = det_mixture(778, 4, 128, 6, 0.5)[0]
    orc, idx = _build_both(e8q, oracle_lib, x, cm, lab, plan_spec="128:0")
    assert idx.plan == [(128, 0)]
    assert idx.bits_per_dim == 0.0
    assert rel_err(idx.estimate(q[0], 3), orc.estimate(q[0], 3)) < 1e-6
    ids, d = idx.search(q, 10, 2, mode="batched")
    oi, od = orc.search(q, 10, 2)
    assert np.allclose(np.sort(d, axis=1), np.sort(od, axis=1), rtol=RTOL, atol=1e-5)


@pytest.mark.parametrize("dim,avg,spec", [(768, 4.0, ""), (320, 3.0, ""), (250, 4.0, "64:3,64:0,128:5")])
def test_me8q_gpu_precision_mode(e8q, oracle_lib, dim, avg, spec):
    """Int8 tensor-core candidates + exact rescoring: recall of the exact
    top-k, and every returned distance is the reference estimator's."""
    n, nlist, nq = 20000, 32, 64
    x, cm, lab = det_mixture(7100 + dim, n, dim, nlist, 0.6)
    q = det_mixture(7200 + dim, nq, dim, nlist, 0.6)[0]
    orc, idx = _build_both(e8q, oracle_lib, x, cm, lab, avg_bits=avg, seed=9, plan_spec=spec)
    for k, nprobe in ((10, 8), (100, 4), (1, 32)):
        ei, ed = idx.search(q, k, nprobe, mode="batched")  # exact grouped scan
        pi, pdd = idx.search(q, k, nprobe, mode="precision")
        oi, od = orc.search(q, k, nprobe)
        hits = sum(len(set(a.tolist()) & set(b.tolist())) for a, b in zip(pi, ei))
        assert hits / ei.size >= 0.97, (k, nprobe, hits / ei.size)
        for r in range(nq):
            ref = {int(i): float(d) for i, d in zip(oi[r], od[r]) if i != 0xFFFFFFFF}
            for i, d in zip(pi[r], pdd[r]):
                if int(i) in ref:
                    assert rel_err(d, ref[int(i)]) < 1e-5, (k, nprobe, r, int(i))
        assert np.all(np.diff(pdd, axis=1) >= 0)
