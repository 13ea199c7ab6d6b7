"""List-sharded search with the CUDA engine: two gloo ranks (CPU collective)
each holding a real E8qIndex / Me8qIndex shard on GPU 0 -- the ranks' kernels
run independently, only their top-k rows meet in the all-gather. The merged
results equal one index over all lists (the oracle's for E8Q, a single GPU
Me8qIndex built with the same variance for ME8Q). The NCCL path is the same
code with the gather and merge on the device; this pool gives one GPU per
run, so it is covered by the merge tests instead."""
import os
import socket

import numpy as np
import pytest

from gen import det_mixture
from parity import assert_topk_parity

pytestmark = pytest.mark.gpu


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, kind, nbits, x, cm, lab, q, k, nprobe, var, ref_ids, ref_d):
    import torch.distributed as dist

    from e8qlib.sharded import ShardedIndex

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sh = ShardedIndex(x.shape[1], nbits, seed=3, device=0, kind=kind)
        if kind == "e8q":
            sh.build(x, cm, lab)
            ids, d = sh.search(q, k, nprobe, mode="plain")
        else:
            sh.build(x, cm, lab, variance=var)
            ids, d = sh.search(q, k, nprobe, mode="batched")
        assert np.nonzero(sh.owner == rank)[0].size > 0
        assert_topk_parity(ids, d, ref_ids, ref_d)
    finally:
        dist.destroy_process_group()


def test_two_rank_e8q_cuda_shards_match_single_index(oracle_lib):
    import torch.multiprocessing as mp

    dim, nlist, k, nprobe, bits = 192, 16, 10, 6, 5
    x, cm, lab = det_mixture(91, 6000, dim, nlist, 0.5)
    q = det_mixture(92, 32, dim, nlist, 0.5)[0]
    single = oracle_lib.OracleE8qIndex(x, cm, lab, bits, seed=3, threads=4)
    ref_ids, ref_d = single.search(q, k, nprobe, threads=4)
    mp.spawn(_worker, args=(2, _port(), "e8q", bits, x, cm, lab, q, k, nprobe, None, ref_ids, ref_d), nprocs=2,
             join=True)


def test_two_rank_me8q_cuda_shards_match_single_index():
    import torch.multiprocessing as mp

    import e8qlib

    dim, nlist, k, nprobe = 256, 16, 10, 6
    x, cm, lab = det_mixture(93, 6000, dim, nlist, 0.5)
    q = det_mixture(94, 32, dim, nlist, 0.5)[0]
    var = x.astype(np.float64).var(axis=0).astype(np.float32)
    single = e8qlib.Me8qIndex(dim, 4.0, 3, device=0)
    single.build(x, cm, lab, variance=var)
    ref_ids, ref_d = single.search(q, k, nprobe, mode="batched")
    del single
    mp.spawn(_worker, args=(2, _port(), "me8q", 4.0, x, cm, lab, q, k, nprobe, var, ref_ids, ref_d), nprocs=2,
             join=True)
