"""GPU parity of the E8Q path against the oracle and the reference's golden
vectors. Everything here runs the CUDA library (libe8qcuda.so) through the
e8qlib Python module, i.e. through the C ABI."""
import numpy as np
import pytest

from conftest import load_golden
from gen import det_mixture, det_normal, det_unit
from parity import assert_topk_parity, rel_err

pytestmark = pytest.mark.gpu

INDEX_CASES = ["d96_b4", "d100_b1", "d128_b9", "d960_b6", "d64_b2_k128"]


@pytest.fixture(scope="module")
def e8q():
    import e8qlib

    return e8qlib


def test_native_library_loaded(e8q):
    import e8qlib._e8qlib as m

    assert m.__file__.endswith(".so")
    assert e8q.version() >= 10000


@pytest.mark.parametrize("pd", [64, 128, 960])
def test_gpu_encoder_bit_exact_golden(e8q, pd):
    g = load_golden("encode.npz")
    rows = {64: 96, 128: 64, 960: 24}[pd]
    u = det_unit(200 + pd, rows, pd)
    for b in range(1, 14):
        dg, br = e8q.encode(u, b)
        assert np.array_equal(dg, g[f"digits_{pd}_b{b}"]), b
        assert np.array_equal(br, g[f"branch_{pd}_b{b}"]), b


def test_gpu_encoder_bit_exact_oracle(e8q, oracle_lib):
    rng = np.random.default_rng(3)
    for pd in (64, 192, 768):
        u = rng.standard_normal((300, pd))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        u = u.astype(np.float32)
        for b in range(1, 14):
            dg, br = e8q.encode(u, b)
            od, ob = oracle_lib.encode(u, b)
            assert np.array_equal(dg, od) and np.array_equal(br, ob), (pd, b)


def test_gpu_rotation_bit_exact(e8q):
    g = load_golden("rotator.npz")
    for dim, seed in [(64, 0), (100, 1), (128, 7), (768, 3), (960, 5)]:
        x = det_normal(100 + dim + seed, (4, dim))
        y = e8q.rotate(x, dim, seed)
        assert np.array_equal(y.view(np.uint32), g[f"rot_{dim}_{seed}"].view(np.uint32)), dim


def test_gpu_rotation_every_width(e8q, oracle_lib):
    """Every padded width of the register-form rotation (64..1024, both FHT
    sizes a width admits) and the shared-memory form around it (dim < 32,
    padded_dim > 1024) agree with the oracle bit for bit."""
    dims = [20, 31, 32, 33, 63, 64, 96, 128, 129, 192, 193, 256, 300, 384, 420, 449, 512, 520, 640, 700,
            768, 800, 896, 930, 960, 961, 1000, 1023, 1024, 1100, 2000]
    for dim in dims:
        seed = dim % 7
        x = det_normal(7000 + dim, (9, dim))
        y = e8q.rotate(x, dim, seed)
        o = oracle_lib.rotate(x, dim, oracle_lib.rotator_signs(dim, seed))
        assert np.array_equal(y.view(np.uint32), o.view(np.uint32)), dim


@pytest.mark.parametrize("name", INDEX_CASES)
def test_gpu_build_matches_reference_index(e8q, name):
    """Codes, ids and the (g1, h3) fit of a GPU-built index equal the
    reference-built index (golden, parsed from its E8AX file)."""
    g = load_golden(f"index_{name}.npz")
    dim, bits, n, nlist, seed, nq, k, nprobe = (int(v) for v in g["params"])
    x, cm, lab = det_mixture(seed, n, dim, nlist, float(g["sigma"]))
    idx = e8q.E8qIndex(dim, bits, seed)
    idx.build(x, cm, lab)
    ids, dg, br, g1, h3 = idx.export_codes()
    assert np.array_equal(ids, g["ids"])
    assert np.array_equal(dg, g["digits"])
    assert np.array_equal(br, g["branch"])
    assert np.all(rel_err(g1, g["g1"]) < 1e-6)
    assert np.all(np.abs(h3 - g["h3"]) <= 1e-6 * np.maximum(1.0, np.abs(g["h3"])))
    assert idx.n == n and idx.num_clusters == nlist and idx.is_built


@pytest.mark.parametrize("name", INDEX_CASES)
def test_gpu_plain_search_matches_reference(e8q, name):
    g = load_golden(f"index_{name}.npz")
    dim, bits, n, nlist, seed, nq, k, nprobe = (int(v) for v in g["params"])
    x, cm, lab = det_mixture(seed, n, dim, nlist, float(g["sigma"]))
    q = det_mixture(seed + 1000, nq, dim, nlist, float(g["sigma"]))[0]
    idx = e8q.E8qIndex(dim, bits, seed)
    idx.build(x, cm, lab)
    ids, dists = idx.search(q, k, nprobe, mode="plain")
    assert ids.dtype == np.uint32 and dists.dtype == np.float32 and ids.shape == (nq, k)
    assert_topk_parity(ids, dists, g["search_ids"], g["search_dists"])
    est = np.array([[idx.estimate(q[i], int(gid)) for gid in g["est_ids"][i]] for i in range(nq)],
                   np.float32)
    ok = np.isfinite(g["est"])
    assert np.all(rel_err(est[ok], g["est"][ok]) < 1e-4)


@pytest.mark.parametrize("dim,bits,nlist,nprobe,k", [
    (128, 4, 32, 8, 10), (960, 6, 16, 4, 10), (768, 4, 24, 24, 100), (200, 5, 20, 64, 32),
    (64, 13, 8, 3, 128), (128, 1, 12, 5, 7), (320, 8, 10, 2, 50), (96, 3, 9, 4, 33)])
def test_gpu_plain_search_vs_oracle(e8q, oracle_lib, dim, bits, nlist, nprobe, k):
    x, cm, lab = det_mixture(dim + bits, 3000, dim, nlist, 0.5)
    q = det_mixture(dim + bits + 7, 25, dim, nlist, 0.5)[0]
    idx = e8q.E8qIndex(dim, bits, 5)
    idx.build(x, cm, lab)
    orc = oracle_lib.OracleE8qIndex(x, cm, lab, bits, seed=5, threads=4)
    ids, dists = idx.search(q, k, nprobe, mode="plain")
    rids, rd = orc.search(q, k, nprobe, threads=4)
    assert_topk_parity(ids, dists, rids, rd)


def test_gpu_edge_cases(e8q, oracle_lib):
    dim, bits = 100, 4
    x, cm, lab = det_mixture(77, 400, dim, 8, 0.5)
    lab = lab.copy()
    lab[lab == 3] = 2                      # list 3 empty
    lab[:33] = 5                           # list 5: >= 33 vectors, spans tiles
    x[40] = cm[lab[40]]                    # a vector on its centroid (rn = 0)
    lab[100] = 7
    lab[lab == 7] = 6
    lab[100] = 7                           # list 7: a single vector
    idx = e8q.E8qIndex(dim, bits, 1)
    idx.build(x, cm, lab)
    orc = oracle_lib.OracleE8qIndex(x, cm, lab, bits, seed=1)
    q = det_normal(5, (9, dim))
    for k, nprobe in [(1, 1), (128, 100), (10, 8), (50, 1)]:
        ids, d = idx.search(q, k, nprobe, mode="plain")
        rids, rd = orc.search(q, k, nprobe)
        assert_topk_parity(ids, d, rids, rd)
    # fewer candidates than k: padding
    for mode in ("plain", "pruned"):
        ids, d = idx.search(q[:2], 128, 1, mode=mode)
        assert np.all(ids[np.isinf(d)] == 0xFFFFFFFF)
    assert idx.estimate(x[40], 40) == pytest.approx(orc.estimate(x[40], 40), rel=1e-4, abs=1e-4)


def test_gpu_errors(e8q):
    with pytest.raises(ValueError):
        e8q.E8qIndex(16, 0)
    with pytest.raises(ValueError):
        e8q.E8qIndex(0, 4)
    idx = e8q.E8qIndex(32, 4)
    with pytest.raises(RuntimeError):
        idx.search(np.zeros((1, 32), np.float32), 1, 1)
    x, cm, lab = det_mixture(3, 200, 32, 4, 0.5)
    with pytest.raises(ValueError):
        idx.build(x, cm, (lab + 10).astype(np.uint32))
    idx.build(x, cm, lab)
    q = x[:2]
    for k, nprobe in [(0, 1), (129, 1), (1, 0)]:
        with pytest.raises(ValueError):
            idx.search(q, k, nprobe)
    with pytest.raises(ValueError):
        idx.search(np.zeros((1, 31), np.float32), 1, 1)
    with pytest.raises(ValueError):
        idx.estimate(q[0], 10**6)
    with pytest.raises(ValueError):
        idx.search(np.zeros(32, np.float32), 1, 1)
