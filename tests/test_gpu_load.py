"""E8qIndex.load on index files written by the reference itself
(tests/golden/index_<name>.e8ax, made by tests/golden/make_golden.py from the
same builds as index_<name>.npz): the loaded device index holds the reference's
codes, g1, h3 and ids bit for bit, and its searches and estimates agree with
the reference's own results. Rates 4, 1 and 9 cover the three split-decode
forms (b = 1 keeps the whole code in the scan byte; b >= 9 fields pass 64 bits)."""
import os

import numpy as np
import pytest

from conftest import ROOT, load_golden
from gen import det_mixture
from parity import assert_topk_parity, rel_err

pytestmark = pytest.mark.gpu

CASES = ["d96_b4", "d100_b1", "d128_b9"]


@pytest.fixture(scope="module")
def e8q():
    import e8qlib

    return e8qlib


def path_of(name):
    return os.path.join(ROOT, "tests", "golden", f"index_{name}.e8ax")


@pytest.mark.parametrize("name", CASES)
def test_load_reference_file(e8q, name):
    G = load_golden(f"index_{name}.npz")
    dim, bits, n, nlist, seed, nq, k, nprobe = (int(v) for v in G["params"])
    idx = e8q.E8qIndex.load(path_of(name))
    assert idx.is_built and idx.dim == dim and idx.nbits == bits
    assert idx.n == n and idx.num_clusters == nlist
    ids, dg, br, g1, h3 = idx.export_codes()
    assert np.array_equal(ids, G["ids"])
    assert np.array_equal(dg, G["digits"]) and np.array_equal(br, G["branch"])
    assert np.array_equal(g1.view(np.uint32), G["g1"].view(np.uint32))
    assert np.array_equal(h3.view(np.uint32), G["h3"].view(np.uint32))
    q = det_mixture(seed + 1000, nq, dim, nlist, float(G["sigma"]))[0]
    for mode in ("plain", "batched"):
        got_ids, got_d = idx.search(q, k, nprobe, mode=mode)
        assert_topk_parity(got_ids, got_d, G["search_ids"], G["search_dists"])
    est = np.array([[idx.estimate(q[i], int(g)) if g != 0xFFFFFFFF else np.nan for g in G["est_ids"][i]]
                    for i in range(nq)], np.float32)
    fin = np.isfinite(G["est"])
    assert rel_err(est[fin], G["est"][fin]).max() < 1e-4


def test_load_matches_gpu_build(e8q):
    """The same data built on the GPU and loaded from the reference's file give
    the same codes and the same results in every mode."""
    G = load_golden("index_d96_b4.npz")
    dim, bits, n, nlist, seed, nq, k, nprobe = (int(v) for v in G["params"])
    x, cm, lab = det_mixture(seed, n, dim, nlist, float(G["sigma"]))
    q = det_mixture(seed + 1000, nq, dim, nlist, float(G["sigma"]))[0]
    built = e8q.E8qIndex(dim, bits, seed)
    built.build(x, cm, lab)
    loaded = e8q.E8qIndex.load(path_of("d96_b4"))
    for a, b in zip(built.export_codes(), loaded.export_codes()):
        assert np.array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8))
    for mode in ("plain", "batched", "precision"):
        ia, da = built.search(q, k, nprobe, mode=mode)
        ib, db = loaded.search(q, k, nprobe, mode=mode)
        assert np.array_equal(ia, ib) and np.array_equal(da.view(np.uint32), db.view(np.uint32)), mode


def test_load_errors(e8q, tmp_path):
    with pytest.raises(RuntimeError, match="cannot open"):
        e8q.E8qIndex.load(str(tmp_path / "missing.e8ax"))
    bad = tmp_path / "foreign.bin"
    bad.write_bytes(b"\x00" * 64)
    with pytest.raises(RuntimeError, match="not an E8Q index"):
        e8q.E8qIndex.load(str(bad))
    raw = open(path_of("d96_b4"), "rb").read()
    cut = tmp_path / "truncated.e8ax"
    cut.write_bytes(raw[: len(raw) // 2])
    with pytest.raises(RuntimeError, match="short read"):
        e8q.E8qIndex.load(str(cut))
