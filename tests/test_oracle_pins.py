"""Pins the CPU oracle (oracle/e8q_oracle.c) to the reference.

Two anchors: the committed golden vectors (tests/golden/*.npz, produced by
running the reference compiled from its own sources; see make_golden.py) and,
when oracle/_ref exists, the live reference itself on fresh inputs.
"""
import hashlib

import numpy as np
import pytest

from conftest import load_golden
from gen import det_mixture, det_normal, det_unit

INDEX_CASES = ["d96_b4", "d100_b1", "d128_b9", "d960_b6", "d64_b2_k128"]


def test_levels_scales_tables(oracle_lib):
    O = oracle_lib
    g = load_golden("levels.npz")
    for b in range(1, 14):
        for br in (0, 1):
            a = O.branch_levels(b, br)
            assert hashlib.sha256(a.tobytes()).digest() == g[f"sha_b{b}_br{br}"].tobytes()
            if b <= 8:
                assert np.array_equal(a, g[f"lev_b{b}_br{br}"])
            # reflection identity, src/.../e8q_test.cpp:35-47
            other = O.branch_levels(b, 1 - br)
            assert np.allclose(other[::-1], -a, atol=1e-9)
        assert O.fixed_scale(b) == float(g[f"scale_b{b}"])
        t = O.refine_tables(b, 960)
        assert hashlib.sha256(t.tobytes()).digest() == g[f"sha_tab_b{b}_pd960"].tobytes()
        w = np.zeros(2)
        O.lib().orc_scan_class_means(b, w)
        assert np.array_equal(w, g[f"wcls_b{b}"])
        assert abs(w[0] + w[1]) < 1e-9


def test_rotator(oracle_lib):
    O = oracle_lib
    g = load_golden("rotator.npz")
    for dim, seed in [(64, 0), (100, 1), (128, 7), (768, 3), (960, 5)]:
        s = O.rotator_signs(dim, seed)
        assert np.array_equal(s, g[f"signs_{dim}_{seed}"])
        x = det_normal(100 + dim + seed, (4, dim))
        y = O.rotate(x, dim, s)
        assert np.array_equal(y.view(np.uint32), g[f"rot_{dim}_{seed}"].view(np.uint32))


@pytest.mark.parametrize("pd", [64, 128, 960])
def test_encoder_bit_exact(oracle_lib, pd):
    O = oracle_lib
    g = load_golden("encode.npz")
    rows = {64: 96, 128: 64, 960: 24}[pd]
    u = det_unit(200 + pd, rows, pd)
    for b in range(1, 14):
        dg, br = O.encode(u, b)
        assert np.array_equal(dg, g[f"digits_{pd}_b{b}"]), b
        assert np.array_equal(br, g[f"branch_{pd}_b{b}"]), b
        # even parity of the digit sum: the E8 quotient shell (e8q_test.cpp:245-279)
        assert np.all((dg.astype(np.int64).sum(-1) & 1) == 0)
        assert dg.max() < (1 << b)


def test_pack_layout(oracle_lib):
    """PackCoarseRow / PackRefineBlock byte layout and the split decode."""
    import ctypes as C

    O = oracle_lib
    L = O.lib()
    g = load_golden("encode.npz")
    for b in range(1, 14):
        dg = g[f"digits_64_b{b}"].reshape(-1, 8)[:64]
        brs = g[f"branch_64_b{b}"].reshape(-1)[:64]
        for i in range(64):
            d = np.ascontiguousarray(dg[i])
            assert L.orc_pack_coarse(d, int(brs[i]), b) == g[f"rowa_b{b}"][i]
            rf = np.zeros(16, np.uint8)
            L.orc_pack_refine(d, int(brs[i]), b, rf)
            assert np.array_equal(rf[: max(b - 1, 0)], g[f"refine_b{b}"][i][: max(b - 1, 0)])
            back = np.zeros(8, np.uint16)
            bro = C.c_int(-1)
            L.orc_decode_split(b, int(g[f"rowa_b{b}"][i]), np.ascontiguousarray(rf), back,
                               C.byref(bro))
            assert np.array_equal(back, d) and bro.value == brs[i]


@pytest.mark.parametrize("name", INDEX_CASES)
def test_index_build_and_plain_search(oracle_lib, name):
    O = oracle_lib
    g = load_golden(f"index_{name}.npz")
    dim, bits, n, nlist, seed, nq, k, nprobe = (int(v) for v in g["params"])
    x, cm, lab = det_mixture(seed, n, dim, nlist, float(g["sigma"]))
    q = det_mixture(seed + 1000, nq, dim, nlist, float(g["sigma"]))[0]
    idx = O.OracleE8qIndex(x, cm, lab, bits, seed=seed, threads=4)
    for f in ("ids", "mean_rot", "centroid_rot", "cn2", "list_begin", "digits", "branch",
              "g1", "h3"):
        a, r = getattr(idx, f), g[f]
        assert np.array_equal(a.reshape(r.shape), r), f
    ids, dists = idx.search(q, k, nprobe, threads=4)
    # plain search: same ids (outside ties), distances within 1e-4 relative
    rel = np.abs(dists - g["search_dists"]) / np.maximum(np.abs(g["search_dists"]), 1e-3)
    finite = np.isfinite(g["search_dists"])
    assert np.all(rel[finite] < 1e-4)
    assert np.array_equal(np.isfinite(dists), finite)
    same = ids == g["search_ids"]
    # any id mismatch must be a near-tie of distances
    for i, j in zip(*np.nonzero(~same)):
        assert abs(float(dists[i, j]) - float(g["search_dists"][i, j])) <= 1e-4 * max(
            1.0, abs(float(g["search_dists"][i, j])))
    est = np.array([[idx.estimate(q[i], int(gid)) for gid in g["est_ids"][i]]
                    for i in range(nq)], np.float32)
    ok = np.isfinite(g["est"])
    assert np.all(np.abs(est[ok] - g["est"][ok]) <= 1e-4 * np.maximum(1.0, np.abs(g["est"][ok])))


def test_live_reference_encoder(oracle_lib):
    """Fresh inputs against the reference compiled here (skipped on machines
    that only carry the committed fixtures)."""
    O = oracle_lib
    if O.ref_lib() is None:
        pytest.skip("reference not built here")
    rng = np.random.default_rng(5)
    for pd in (64, 192, 768):
        u = rng.standard_normal((40, pd))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        u = u.astype(np.float32)
        for b in range(1, 14):
            a = O.encode(u, b)
            r = O.ref_encode(u, b)
            assert np.array_equal(a[0], r[0]) and np.array_equal(a[1], r[1]), (pd, b)
