"""Generate the golden fixtures in tests/golden/ by RUNNING THE REFERENCE.

Needs the reference compiled from its own sources (``make -C oracle ref``,
which reads the reference tree). Inputs come from tests/golden/gen.py (exact
integer-derived floats), outputs come from the reference's own code:
  * oracle/_ref/libe8qref.so  - BranchLevels, FixedScale, EncodeVectorAtScale,
    BuildRefineTables, PackCoarseRow/PackRefineBlock, FhtKac4Rotator
  * oracle/_ref/e8qlib_ref    - the reference's pybind11 module: E8qIndex
    build / save (E8AX, parsed for codes, g1, h3, ids) / plain search
    (set_disable_prune(True)) / estimate / production pruned search with its
    per-query stats; Me8qIndex build / save / search (prune_alpha 1e-9: the
    plain scan) and its production FastScan search with per-query stats.

Usage: python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)

import oracle as O  # noqa: E402
from gen import det_mixture, det_normal, det_unit  # noqa: E402

ROT_CASES = [(64, 0), (100, 1), (128, 7), (768, 3), (960, 5)]
ENC_DIMS = [64, 128, 960]
ENC_ROWS = {64: 96, 128: 64, 960: 24}
# (name, dim, bits, n, nlist, seed, sigma, nq, k, nprobe)
INDEX_CASES = [
    ("d96_b4", 96, 4, 1500, 8, 11, 0.5, 20, 10, 3),
    ("d100_b1", 100, 1, 800, 4, 12, 0.5, 12, 10, 2),
    ("d128_b9", 128, 9, 600, 4, 13, 0.5, 12, 16, 4),
    ("d960_b6", 960, 6, 300, 4, 14, 0.4, 8, 10, 2),
    ("d64_b2_k128", 64, 2, 700, 5, 15, 0.5, 6, 128, 5),
]
# ME8Q: (name, dim, avg_bits, seed, plan_spec, n, nlist, sigma, nq, k, nprobe)
ME8Q_CASES = [
    ("me8q_d200_spec", 200, 4.0, 0, "64:6,64:4,64:3,64:0", 1500, 12, 0.5, 10, 10, 5),
    ("me8q_d200_a4", 200, 4.0, 7, "", 1500, 12, 0.5, 10, 10, 5),
    ("me8q_d150_a3", 150, 3.0, 0, "", 1200, 10, 0.5, 8, 16, 4),
    ("me8q_d96_a6", 96, 6.0, 11, "", 900, 8, 0.5, 8, 10, 3),
]


# reference-written E8AX index files, kept whole, for the loader's tests
E8AX_FILES = ["d96_b4", "d100_b1", "d128_b9"]


# the reference's shipped pruned search, query by query with its stats:
# (name, dim, bits, n, nlist, seed, sigma, nq, k, nprobe, alpha)
PRUNED_CASES = [
    ("d96_b4", 96, 4, 1500, 8, 11, 0.5, 20, 10, 3, 1.0),
    ("d100_b1", 100, 1, 800, 4, 12, 0.5, 12, 10, 2, 1.0),
    ("d128_b9", 128, 9, 600, 4, 13, 0.5, 12, 16, 4, 1.0),
    ("d960_b6", 960, 6, 3000, 8, 14, 0.4, 16, 10, 3, 1.0),
    ("d64_b2_k128", 64, 2, 2000, 6, 15, 0.5, 12, 128, 5, 1.0),
    ("d200_b5_a001", 200, 5, 4000, 16, 16, 0.5, 16, 10, 6, 0.01),
]


def write_pruned_fixtures() -> None:
    """The reference's production (pruned) search on PRUNED_CASES, one call
    per query with return_stats so each query's candidate and survivor counts
    are kept (tests/golden/pruned_<name>.npz), plus its scan-bank headers."""
    import oracle as O

    E = O.ref_module()
    for name, dim, bits, n, nlist, seed, sigma, nq, k, nprobe, alpha in PRUNED_CASES:
        x, cm, lab = det_mixture(seed, n, dim, nlist, sigma)
        q = det_mixture(seed + 1000, nq, dim, nlist, sigma)[0]
        idx = E.E8qIndex(dim, bits, seed)
        idx.build(x, cm, lab, num_threads=4, prune_alpha=alpha)
        with tempfile.TemporaryDirectory() as d:
            p = os.path.join(d, "i.e8ax")
            idx.save(p)
            P = O.parse_e8ax(p)
        ids, dists, cand, surv = [], [], [], []
        for i in range(nq):
            a, b, st = idx.search(q[i:i + 1], k, nprobe, 1, True)
            ids.append(a[0])
            dists.append(b[0])
            cand.append(st["candidates"])
            surv.append(st["survivors"])
        np.savez_compressed(
            os.path.join(HERE, f"pruned_{name}.npz"),
            params=np.array([dim, bits, n, nlist, seed, nq, k, nprobe], np.int64),
            sigma=np.float64(sigma), alpha=np.float32(alpha), banks=P["banks"],
            search_ids=np.array(ids, np.uint32), search_dists=np.array(dists, np.float32),
            candidates=np.array(cand, np.uint64), survivors=np.array(surv, np.uint64))


# (name, dim, bits, n, nlist, seed, sigma, nq, pairs)
PROBE_CASES = [
    ("d96_b4", 96, 4, 3000, 20, 31, 0.5, 8, 64),
    ("d100_b1", 100, 1, 2000, 16, 32, 0.5, 6, 48),
    ("d200_b9", 200, 9, 2500, 24, 33, 0.45, 5, 40),
]


def write_probe_fixtures() -> None:
    """The reference's E8qIndex.probe_bound_w on PROBE_CASES: pair i probes
    stored vector ids[i] (its raw row as base) with query qidx[i]
    (tests/golden/probe_bound_<name>.npz)."""
    import oracle as O

    E = O.ref_module()
    for name, dim, bits, n, nlist, seed, sigma, nq, pairs in PROBE_CASES:
        x, cm, lab = det_mixture(seed, n, dim, nlist, sigma)
        q = det_mixture(seed + 1000, nq, dim, nlist, sigma)[0]
        idx = E.E8qIndex(dim, bits, seed)
        idx.build(x, cm, lab, num_threads=4)
        rng = np.random.default_rng(seed)
        ids = rng.choice(n, pairs, replace=False).astype(np.uint32)
        qidx = rng.integers(0, nq, pairs).astype(np.uint32)
        out = idx.probe_bound_w(q, x[ids], qidx, ids)
        np.savez_compressed(os.path.join(HERE, f"probe_bound_{name}.npz"),
                            params=np.array([dim, bits, n, nlist, seed, nq], np.int64), sigma=np.float64(sigma),
                            ids=ids, qidx=qidx, out=np.asarray(out, np.float64))


# the reference's production ME8Q search (FastScan cascade), query by query
# with its stats: (name, dim, avg_bits, seed, plan_spec, n, nlist, sigma, nq,
# k, nprobe, prune_alpha)
ME8Q_PRUNED_CASES = [
    ("d200_a4", 200, 4.0, 7, "", 3000, 12, 0.5, 24, 10, 5, 0.0),
    ("d200_spec", 200, 4.0, 0, "64:6,64:4,64:3,64:0", 3000, 12, 0.5, 24, 10, 5, 0.0),
    ("d96_a6_k20", 96, 6.0, 11, "", 2500, 8, 0.5, 24, 20, 3, 0.0),
    ("d150_a3_a001", 150, 3.0, 0, "", 4000, 10, 0.5, 24, 16, 4, 0.01),
    ("d64_a1", 64, 1.0, 3, "", 2000, 6, 0.5, 16, 10, 3, 0.0),
    ("d192_k100_np_all", 192, 3.0, 5, "", 3000, 8, 0.5, 12, 100, 20, 0.0),
    ("d256_spec_r1", 256, 3.0, 9, "64:5,64:1,64:3,64:0", 3500, 10, 0.5, 16, 16, 4, 0.3),
]


def write_me8q_pruned_fixtures() -> None:
    """The reference's Me8qIndex.search (its only search: the FastScan
    cascade) on ME8Q_PRUNED_CASES, one call per query with return_stats
    (tests/golden/me8q_pruned_<name>.npz)."""
    import oracle as O

    E = O.ref_module()
    for name, dim, avg, seed, spec, n, nlist, sigma, nq, k, nprobe, alpha in ME8Q_PRUNED_CASES:
        x, cm, lab = det_mixture(seed + 5000 + dim, n, dim, nlist, sigma)
        q = det_mixture(seed + 6000 + dim, nq, dim, nlist, sigma)[0]
        idx = E.Me8qIndex(dim, avg, seed)
        idx.build(x, cm, lab, num_threads=1, plan_spec=spec, prune_alpha=alpha)
        ids, dists, cand, surv = [], [], [], []
        for i in range(nq):
            a, b, st = idx.search(q[i:i + 1], k, nprobe, 1, True)
            ids.append(a[0])
            dists.append(b[0])
            cand.append(st["candidates"])
            surv.append(st["survivors"])
        np.savez_compressed(
            os.path.join(HERE, f"me8q_pruned_{name}.npz"),
            params=np.array([dim, seed, n, nlist, nq, k, nprobe], np.int64), avg_bits=np.float64(avg),
            sigma=np.float64(sigma), plan_spec=np.array(spec), alpha=np.float32(alpha),
            search_ids=np.array(ids, np.uint32), search_dists=np.array(dists, np.float32),
            candidates=np.array(cand, np.uint64), survivors=np.array(surv, np.uint64))


# reference-written ME8QIDXX index files, kept whole, for the ME8Q loader's tests
ME8Q_FILES = ["me8q_d200_spec", "me8q_d150_a3"]


def write_me8q_fixtures() -> None:
    """Build the ME8Q_FILES cases of ME8Q_CASES with the reference (one thread,
    as the parsed fixtures) and keep its saved index files
    (tests/golden/<name>.me8q)."""
    import oracle as O

    E = O.ref_module()
    for name, dim, avg, seed, spec, n, nlist, sigma, nq, k, nprobe in ME8Q_CASES:
        if name not in ME8Q_FILES:
            continue
        x, cm, lab = det_mixture(seed + 5000 + dim, n, dim, nlist, sigma)
        idx = E.Me8qIndex(dim, avg, seed)
        idx.build(x, cm, lab, num_threads=1, plan_spec=spec, prune_alpha=1e-9)
        idx.save(os.path.join(HERE, f"{name}.me8q"))


def write_e8ax_fixtures() -> None:
    """Build the E8AX_FILES cases of INDEX_CASES with the reference and keep
    its saved index files (tests/golden/index_<name>.e8ax): the same builds
    whose parsed contents and search results are in index_<name>.npz."""
    import oracle as O

    E = O.ref_module()
    for name, dim, bits, n, nlist, seed, sigma, nq, k, nprobe in INDEX_CASES:
        if name not in E8AX_FILES:
            continue
        x, cm, lab = det_mixture(seed, n, dim, nlist, sigma)
        idx = E.E8qIndex(dim, bits, seed)
        idx.build(x, cm, lab, num_threads=4)
        idx.save(os.path.join(HERE, f"index_{name}.e8ax"))


def main() -> None:
    R = O.ref_lib()
    E = O.ref_module()
    if R is None or E is None:
        raise SystemExit("build the reference first: make -C oracle ref")

    # ---- levels, scales, refine tables --------------------------------
    lv = {}
    for b in range(1, 14):
        for br in (0, 1):
            a = np.zeros(1 << b, np.float64)
            R.ref_branch_levels(b, br, a)
            lv[f"sha_b{b}_br{br}"] = np.frombuffer(hashlib.sha256(a.tobytes()).digest(), np.uint8)
            if b <= 8:
                lv[f"lev_b{b}_br{br}"] = a
        lv[f"scale_b{b}"] = np.float64(R.ref_fixed_scale(b))
        t = np.zeros(2 * max(256, 1 << b), np.float32)
        R.ref_refine_tables(b, 960, t)
        lv[f"sha_tab_b{b}_pd960"] = np.frombuffer(hashlib.sha256(t.tobytes()).digest(), np.uint8)
        w = np.zeros(2, np.float64)
        R.ref_scan_class_means(b, w)
        lv[f"wcls_b{b}"] = w
    np.savez_compressed(os.path.join(HERE, "levels.npz"), **lv)

    # ---- rotator -------------------------------------------------------
    rot = {}
    for dim, seed in ROT_CASES:
        nb = R.ref_rotator_sign_bytes(dim, seed)
        s = np.zeros(nb, np.uint8)
        R.ref_rotator_signs(dim, seed, s)
        x = det_normal(100 + dim + seed, (4, dim))
        y = np.zeros((4, O.padded_dim(dim)), np.float32)
        R.ref_rotate(dim, seed, x, 4, y)
        rot[f"signs_{dim}_{seed}"] = s
        rot[f"rot_{dim}_{seed}"] = y
    np.savez_compressed(os.path.join(HERE, "rotator.npz"), **rot)

    # ---- encoder -------------------------------------------------------
    enc = {}
    for pd in ENC_DIMS:
        u = det_unit(200 + pd, ENC_ROWS[pd], pd)
        for b in range(1, 14):
            dg, br = O.ref_encode(u, b)
            enc[f"digits_{pd}_b{b}"] = dg
            enc[f"branch_{pd}_b{b}"] = br
    # packed blocks (reference on-disk layout) for the first rows at pd=64
    for b in range(1, 14):
        dg = enc[f"digits_64_b{b}"].reshape(-1, 8)[:64]
        brs = enc[f"branch_64_b{b}"].reshape(-1)[:64]
        rowa = np.zeros(64, np.uint8)
        refine = np.zeros((64, 16), np.uint8)
        for i in range(64):
            ra = np.zeros(1, np.uint8)
            rf = np.zeros(16, np.uint8)
            R.ref_pack_block(np.ascontiguousarray(dg[i]), int(brs[i]), b, ra, rf)
            rowa[i] = ra[0]
            refine[i] = rf
        enc[f"rowa_b{b}"] = rowa
        enc[f"refine_b{b}"] = refine
    np.savez_compressed(os.path.join(HERE, "encode.npz"), **enc)

    # ---- whole indexes -------------------------------------------------
    for name, dim, bits, n, nlist, seed, sigma, nq, k, nprobe in INDEX_CASES:
        x, cm, lab = det_mixture(seed, n, dim, nlist, sigma)
        q = det_mixture(seed + 1000, nq, dim, nlist, sigma)[0]
        idx = E.E8qIndex(dim, bits, seed)
        idx.build(x, cm, lab, num_threads=4)
        idx.set_disable_prune(True)
        with tempfile.TemporaryDirectory() as d:
            p = os.path.join(d, "i.e8ax")
            idx.save(p)
            P = O.parse_e8ax(p)
        ids, dists = idx.search(q, k, nprobe, 1)
        est_ids = ids[:, :3].astype(np.uint32)
        est = np.array([[idx.estimate(q[i], int(g)) if g != 0xFFFFFFFF else np.nan
                         for g in est_ids[i]] for i in range(nq)], np.float32)
        np.savez_compressed(
            os.path.join(HERE, f"index_{name}.npz"),
            params=np.array([dim, bits, n, nlist, seed, nq, k, nprobe], np.int64),
            sigma=np.float64(sigma),
            ids=P["ids"], mean_rot=P["mean_rot"], centroid_rot=P["centroid_rot"], cn2=P["cn2"],
            list_begin=P["list_begin"], digits=P["digits"], branch=P["branch"], g1=P["g1"],
            h3=P["h3"], rowa=P["rowa"], refine=P["refine"], signs=P["signs"],
            search_ids=ids, search_dists=dists, est_ids=est_ids, est=est,
            memory_bytes=np.int64(idx.memory_bytes))
    # ---- ME8Q indexes (single-threaded reference build: its 4-thread build
    # differed on one block of one row in a probe, so the pinned fixtures come
    # from one thread; prune_alpha 1e-9 makes its search the plain scan) -------
    for name, dim, avg, seed, spec, n, nlist, sigma, nq, k, nprobe in ME8Q_CASES:
        x, cm, lab = det_mixture(seed + 5000 + dim, n, dim, nlist, sigma)
        q = det_mixture(seed + 6000 + dim, nq, dim, nlist, sigma)[0]
        idx = E.Me8qIndex(dim, avg, seed)
        idx.build(x, cm, lab, num_threads=1, plan_spec=spec, prune_alpha=1e-9)
        with tempfile.TemporaryDirectory() as d:
            pth = os.path.join(d, "i.me8q")
            idx.save(pth)
            P = O.parse_me8q(pth)
        ids, dists = idx.search(q, k, nprobe, 1)
        est_ids = np.arange(0, n, max(1, n // 25), dtype=np.uint32)
        est = np.array([[idx.estimate(q[i], int(g)) for g in est_ids] for i in range(nq)], np.float32)
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"),
            params=np.array([dim, seed, n, nlist, nq, k, nprobe], np.int64), avg_bits=np.float64(avg),
            sigma=np.float64(sigma), plan_spec=np.array(spec), plan=np.array(P["plan"], np.int64),
            ids=P["ids"], list_begin=P["list_begin"], digits=P["digits"], branch=P["branch"], coef=P["coef"],
            h2=P["h2"], search_ids=ids, search_dists=dists, est_ids=est_ids, est=est)
    write_e8ax_fixtures()
    write_me8q_fixtures()
    write_pruned_fixtures()
    write_me8q_pruned_fixtures()
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "e8ax":
        write_e8ax_fixtures()  # only the E8AX files
    elif len(sys.argv) > 1 and sys.argv[1] == "me8q":
        write_me8q_fixtures()  # only the ME8QIDXX files
    elif len(sys.argv) > 1 and sys.argv[1] == "probe":
        write_probe_fixtures()
    elif len(sys.argv) > 1 and sys.argv[1] == "pruned":
        write_pruned_fixtures()  # only the pruned-search fixtures
    elif len(sys.argv) > 1 and sys.argv[1] == "me8q_pruned":
        write_me8q_pruned_fixtures()  # only the ME8Q production-search fixtures
    else:
        main()
