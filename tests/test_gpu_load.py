"""E8qIndex.load and Me8qIndex.load on index files written by the reference
itself (tests/golden/index_<name>.e8ax and <name>.me8q, made by
tests/golden/make_golden.py from the same builds as the .npz fixtures): the
loaded device index holds the reference's codes and factors and ids bit for
bit, and its searches and estimates agree with the reference's own results.
E8Q rates 4, 1 and 9 cover the three split-decode forms (b = 1 keeps the whole
code in the scan byte; b >= 9 fields pass 64 bits); the ME8Q files cover a
manual plan with a dropped run and a DP plan."""
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


ME8Q_CASES = ["me8q_d200_spec", "me8q_d150_a3"]


@pytest.mark.parametrize("name", ME8Q_CASES)
def test_me8q_load_reference_file(e8q, name):
    """Me8qIndex.load on a file the reference wrote: plan, ids, every segment
    code and (coef, h2) bit for bit, estimates and the plain search as the
    reference's own (the same build as me8q_<name>.npz)."""
    G = load_golden(name + ".npz")
    dim, seed, n, nlist, nq, k, nprobe = (int(v) for v in G["params"])
    m = e8q.Me8qIndex.load(os.path.join(ROOT, "tests", "golden", f"{name}.me8q"))
    assert m.is_built and m.dim == dim and m.n == n and m.num_clusters == nlist
    assert [list(p) for p in m.plan] == [list(p) for p in G["plan"]]
    assert m.avg_bits == pytest.approx(m.bits_per_dim)
    ids, dg, br, cf, h2 = m.export_codes()
    assert np.array_equal(ids, G["ids"])
    assert np.array_equal(dg, G["digits"]) and np.array_equal(br, G["branch"])
    assert np.array_equal(cf.view(np.uint32), G["coef"].view(np.uint32))
    assert np.array_equal(h2.view(np.uint32), G["h2"].view(np.uint32))
    q = det_mixture(seed + 6000 + dim, nq, dim, nlist, float(G["sigma"]))[0]
    est = np.array([[m.estimate(q[i], int(g)) for g in G["est_ids"]] for i in range(nq)], np.float32)
    assert rel_err(est, G["est"]).max() < 1e-6
    got_ids, got_d = m.search(q, k, nprobe)
    assert_topk_parity(got_ids, got_d, G["search_ids"], G["search_dists"])
    p_ids, p_d = m.search(q, k, nprobe, mode="precision")
    assert p_ids.shape == got_ids.shape and np.all(np.diff(p_d, axis=1) >= 0)


def test_me8q_load_errors(e8q, tmp_path):
    with pytest.raises(RuntimeError, match="cannot read"):
        e8q.Me8qIndex.load(str(tmp_path / "missing.me8q"))
    bad = tmp_path / "foreign.bin"
    bad.write_bytes(b"\x00" * 64)
    with pytest.raises(RuntimeError, match="bad magic"):
        e8q.Me8qIndex.load(str(bad))
    raw = open(os.path.join(ROOT, "tests", "golden", "me8q_d150_a3.me8q"), "rb").read()
    cut = tmp_path / "truncated.me8q"
    cut.write_bytes(raw[: len(raw) // 2])
    with pytest.raises(RuntimeError, match="short read"):
        e8q.Me8qIndex.load(str(cut))


def test_me8q_save_round_trip_and_reference_load(e8q, oracle_lib, tmp_path):
    """Me8qIndex.save writes what the reference reads: the file parses to the
    reference's own fixture (the same build), loads back on the GPU bit for
    bit, and the reference's Me8qIndex.load accepts it and searches like the
    GPU index."""
    name = "me8q_d200_spec"
    G = load_golden(name + ".npz")
    dim, seed, n, nlist, nq, k, nprobe = (int(v) for v in G["params"])
    x, cm, lab = det_mixture(seed + 5000 + dim, n, dim, nlist, float(G["sigma"]))
    q = det_mixture(seed + 6000 + dim, nq, dim, nlist, float(G["sigma"]))[0]
    m = e8q.Me8qIndex(dim, float(G["avg_bits"]), seed)
    m.build(x, cm, lab, plan_spec=str(G["plan_spec"]), prune_alpha=1e-9)
    path = str(tmp_path / "gpu.me8q")
    m.save(path)
    P = oracle_lib.parse_me8q(path)
    for key in ("ids", "digits", "branch", "coef", "h2"):
        assert np.array_equal(np.asarray(P[key]).view(np.uint8), np.asarray(G[key]).view(np.uint8)), key
    back = e8q.Me8qIndex.load(path)
    for a, b in zip(m.export_codes(), back.export_codes()):
        assert np.array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8))
    assert_topk_parity(*back.search(q, k, nprobe), G["search_ids"], G["search_dists"])
    E = oracle_lib.ref_module()  # the reference compiled into oracle/_ref, present wherever it was built
    if E is not None:
        ref = E.Me8qIndex.load(path)
        rid, rd = ref.search(q, k, nprobe, 1)
        gid, gd = m.search(q, k, nprobe)
        assert_topk_parity(gid, gd, rid, rd)


@pytest.mark.parametrize("name", CASES)
def test_save_matches_reference_file(e8q, name, tmp_path):
    """E8qIndex.save of a GPU-built index writes the reference's own file for
    the same build byte for byte (codes, fits, scan-bank headers, layout,
    trailer); a loaded reference file saves back to itself."""
    G = load_golden(f"index_{name}.npz")
    dim, bits, n, nlist, seed, nq, k, nprobe = (int(v) for v in G["params"])
    x, cm, lab = det_mixture(seed, n, dim, nlist, float(G["sigma"]))
    ref = open(path_of(name), "rb").read()
    built = e8q.E8qIndex(dim, bits, seed)
    built.build(x, cm, lab)
    out = tmp_path / "gpu.e8ax"
    built.save(str(out))
    mine = out.read_bytes()
    assert len(mine) == len(ref)
    diff = np.flatnonzero(np.frombuffer(mine, np.uint8) != np.frombuffer(ref, np.uint8))
    assert diff.size == 0, f"{diff.size} bytes differ, first at {diff[:8]}"
    loaded = e8q.E8qIndex.load(path_of(name))
    again = tmp_path / "again.e8ax"
    loaded.save(str(again))
    assert again.read_bytes() == ref


def test_save_errors(e8q, tmp_path):
    idx = e8q.E8qIndex(32, 4)
    with pytest.raises(RuntimeError):
        idx.save(str(tmp_path / "unbuilt.e8ax"))
    x, cm, lab = det_mixture(3, 200, 32, 4, 0.5)
    idx.build(x, cm, lab)
    with pytest.raises(RuntimeError, match="cannot open"):
        idx.save(str(tmp_path / "no_such_dir" / "x.e8ax"))
