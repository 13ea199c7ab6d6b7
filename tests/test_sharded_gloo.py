"""List-sharded search (e8qlib.sharded) on CPU: partitioning, the top-k merge,
and a world_size-2 gloo run whose merged results match one index over all
lists. The oracle stands in for each rank's GPU index, so only the host-side
sharding and the collective are under test here."""
import os
import socket

import numpy as np
import pytest

from gen import det_mixture
from parity import assert_topk_parity

from e8qlib.sharded import merge_topk, partition_lists

UMAX = 0xFFFFFFFF


def test_partition_balances_and_is_deterministic():
    sizes = [50, 10, 40, 30, 30, 20, 0, 5]
    own = partition_lists(sizes, 3)
    assert own.tolist() == partition_lists(sizes, 3).tolist()
    loads = np.bincount(own, weights=sizes, minlength=3)
    assert loads.max() - loads.min() <= max(sizes)
    assert set(own.tolist()) <= {0, 1, 2}
    assert partition_lists(sizes, 1).tolist() == [0] * len(sizes)


def test_merge_order_ties_and_padding():
    a_i = np.array([[3, 7, UMAX]], np.uint32)
    a_d = np.array([[1.0, 2.0, np.inf]], np.float32)
    b_i = np.array([[5, 2, 9]], np.uint32)
    b_d = np.array([[1.0, 2.0, 3.0]], np.float32)
    ids, d = merge_topk([a_i, b_i], [a_d, b_d], 5)
    assert ids.tolist() == [[3, 5, 2, 7, 9]]
    assert d.tolist() == [[1.0, 1.0, 2.0, 2.0, 3.0]]
    ids, d = merge_topk([a_i[:, :1]], [a_d[:, :1]], 3)
    assert ids.tolist() == [[3, UMAX, UMAX]] and np.isinf(d[0, 1:]).all()


class OracleEngine:
    """The oracle restatement as a rank's engine (CPU)."""

    def __init__(self, bits, seed):
        self.bits, self.seed = bits, seed

    def build(self, data, centroids, cluster_ids):
        import oracle

        self.o = oracle.OracleE8qIndex(data, centroids, cluster_ids, self.bits, seed=self.seed, threads=2)

    def search(self, q, k, nprobe):
        return self.o.search(q, k, nprobe, threads=2)


def _worker(rank, world, port, x, cm, lab, q, k, nprobe, ref_ids, ref_d):
    import torch.distributed as dist

    from e8qlib.sharded import ShardedIndex

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sh = ShardedIndex(x.shape[1], 5, seed=3, make_engine=lambda: OracleEngine(5, 3))
        sh.build(x, cm, lab)
        owned = np.nonzero(sh.owner == rank)[0]
        assert owned.size > 0
        ids, d = sh.search(q, k, nprobe)
        assert_topk_parity(ids, d, ref_ids, ref_d)
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_matches_single_index(oracle_lib):
    import torch.multiprocessing as mp

    dim, nlist, k, nprobe = 96, 12, 10, 5
    x, cm, lab = det_mixture(77, 2400, dim, nlist, 0.5)
    q = det_mixture(78, 40, dim, nlist, 0.5)[0]
    single = oracle_lib.OracleE8qIndex(x, cm, lab, 5, seed=3, threads=2)
    ref_ids, ref_d = single.search(q, k, nprobe, threads=2)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.spawn(_worker, args=(2, port, x, cm, lab, q, k, nprobe, ref_ids, ref_d), nprocs=2, join=True)


def test_vectorised_merges_agree():
    """The host merge (numpy) and the device merge (torch, here on CPU
    tensors) give the same rows: (distance, id) order, -0 == +0, negative
    distances, padding last."""
    import torch

    from e8qlib.sharded import merge_topk_torch

    rng = np.random.default_rng(4)
    nq, m, k = 9, 3, 7
    parts_i, parts_d = [], []
    for r in range(m):
        d = np.sort(rng.choice(np.array([-1.5, -0.0, 0.0, 0.25, 1.0, 2.0, np.inf], np.float32), (nq, k)), axis=1)
        i = rng.permutation(10_000)[:nq * k].reshape(nq, k).astype(np.uint32) + np.uint32(r * 10_000)
        i[np.isinf(d)] = UMAX
        parts_i.append(i)
        parts_d.append(d.astype(np.float32))
    hi, hd = merge_topk(parts_i, parts_d, k)
    ti = torch.from_numpy(np.concatenate(parts_i, 1).view(np.int32))
    td = torch.from_numpy(np.concatenate(parts_d, 1))
    di, dd = merge_topk_torch(ti, td, k)
    assert np.array_equal(di.numpy().view(np.uint32), hi)
    assert np.array_equal(dd.numpy(), hd + np.float32(0.0))
    # reference order by a plain sort of (distance, id) pairs
    for q in range(nq):
        pairs = sorted(zip((np.concatenate(parts_d, 1)[q] + np.float32(0)).tolist(),
                           np.concatenate(parts_i, 1)[q].tolist()))[:k]
        assert [p[1] for p in pairs] == hi[q].tolist()
