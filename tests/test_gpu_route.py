"""Batch routing on the int8 tensor cores (batches of 256 queries or more)
selects the probes of the fp64 route bit for bit: the same queries searched as
one batch and as batches below that size return identical ids and distances,
in every mode that routes a batch, with exact ties (duplicate centroids), a
zero query, a query on a centroid and queries of extreme magnitude."""
import numpy as np
import pytest

from gen import det_mixture

pytestmark = pytest.mark.gpu

SMALL = 200  # below the tensor-core routing threshold (256 queries)


@pytest.fixture(scope="module")
def e8q():
    import e8qlib

    return e8qlib


def edge_queries(q, cm):
    q = q.copy()
    q[0] = 0.0
    q[1] = cm[5]
    q[2] *= 1e6
    q[3] *= 1e-6
    q[4] = 0.5 * (cm[3] + cm[10])
    return q


def split_search(idx, q, ks, nps, k_max, mode):
    parts = [idx.search_ragged(q[i:i + SMALL], ks[i:i + SMALL], nps[i:i + SMALL], k_max, mode=mode)
             for i in range(0, len(q), SMALL)]
    return np.concatenate([p[0] for p in parts]), np.concatenate([p[1] for p in parts])


@pytest.mark.parametrize("dim,nlist", [(200, 48), (960, 130)])
def test_tc_route_matches_fp64_route(e8q, dim, nlist):
    x, cm, lab = det_mixture(71 + dim, 6000, dim, nlist, 0.5)
    cm = cm.copy()
    cm[7] = cm[3]  # identical centroids: equal d2, ties broken by list id
    idx = e8q.E8qIndex(dim, 4, 3)
    idx.build(x, cm, lab)
    q = edge_queries(det_mixture(72 + dim, 600, dim, nlist, 0.5)[0], cm)
    rng = np.random.default_rng(dim)
    ks = rng.integers(1, 33, len(q)).astype(np.uint32)
    nps = rng.integers(1, nlist + 1, len(q)).astype(np.uint32)
    for mode in ("batched", "precision"):
        ids, d = idx.search_ragged(q, ks, nps, 32, mode=mode)
        sids, sd = split_search(idx, q, ks, nps, 32, mode)
        assert np.array_equal(ids, sids), mode
        assert np.array_equal(d.view(np.uint32), sd.view(np.uint32)), mode


def test_tc_route_me8q(e8q):
    dim, nlist = 256, 40
    x, cm, lab = det_mixture(81, 5000, dim, nlist, 0.5)
    m = e8q.Me8qIndex(dim, 4.0, 1)
    m.build(x, cm, lab)
    q = edge_queries(det_mixture(82, 520, dim, nlist, 0.5)[0], cm)
    rng = np.random.default_rng(5)
    ks = rng.integers(1, 17, len(q)).astype(np.uint32)
    nps = rng.integers(1, nlist + 1, len(q)).astype(np.uint32)
    for mode in ("batched", "precision"):
        ids, d = m.search_ragged(q, ks, nps, 16, mode=mode)
        sids, sd = split_search(m, q, ks, nps, 16, mode)
        assert np.array_equal(ids, sids), mode
        assert np.array_equal(d.view(np.uint32), sd.view(np.uint32)), mode


def test_host_and_device_queries_agree(e8q):
    """A 4,100-query batch searched from host memory (staged by the library)
    and from device memory returns the same ids and distances."""
    import torch

    dim, nlist = 128, 32
    x, cm, lab = det_mixture(91, 3000, dim, nlist, 0.5)
    idx = e8q.E8qIndex(dim, 5, 2)
    idx.build(x, cm, lab)
    q = det_mixture(92, 4100, dim, nlist, 0.5)[0]
    qd = torch.from_numpy(q).cuda()
    for mode in ("batched", "precision"):
        ids, d = idx.search(q, 10, 8, mode=mode)
        oi = torch.empty(len(q), 10, dtype=torch.int32, device="cuda")
        od = torch.empty(len(q), 10, dtype=torch.float32, device="cuda")
        idx.search_ptr(qd.data_ptr(), len(q), 10, 8, oi.data_ptr(), od.data_ptr(), mode=mode)
        torch.cuda.synchronize()
        assert np.array_equal(ids.view(np.int32), oi.cpu().numpy()), mode
        assert np.array_equal(d.view(np.uint32), od.cpu().numpy().view(np.uint32)), mode
