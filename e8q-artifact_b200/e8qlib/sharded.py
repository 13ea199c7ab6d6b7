"""List-sharded E8Q search across GPUs: one process per GPU, IVF lists
partitioned over the ranks, one exchange step.

Lists are independent, so each rank holds the vectors of the lists it owns
(all centroids are replicated, so every rank routes a query to the same
probes; lists it does not own are empty locally) and scans only those. The
one collective is an all-gather of every rank's local top-k (distance, id)
per query; the merge keeps the k best under the reference's total order --
smaller distance first, ties by smaller id (src/index/e8q_internal.hpp:47-49),
padding (UINT32_MAX, +inf) last.

Each rank centres its own vectors on their own mean; the estimator's residual
to the list centroid does not depend on that mean, so sharded distances match
a single index's up to float rounding.

The per-rank engine is any object with ``build(data, centroids, cluster_ids)``
and ``search(queries, k, nprobe) -> (ids, dists)``; by default an
``e8qlib.E8qIndex`` on this rank's GPU.
"""
from __future__ import annotations

import numpy as np

UINT32_MAX = np.uint32(0xFFFFFFFF)


def partition_lists(list_sizes, world: int) -> np.ndarray:
    """Owner rank of each list: largest list first onto the least-loaded rank
    (ties: lower rank), so ranks hold about the same number of vectors."""
    sizes = np.asarray(list_sizes, np.int64)
    owner = np.zeros(sizes.shape[0], np.int32)
    load = np.zeros(world, np.int64)
    for c in sorted(range(sizes.shape[0]), key=lambda i: (-sizes[i], i)):
        r = int(np.argmin(load))
        owner[c] = r
        load[r] += sizes[c]
    return owner


def merge_topk(ids_parts, dists_parts, k: int):
    """Merge per-rank top-k rows ([world, nq, k] each) into the global top-k
    under (distance, id) order; padding entries sort last."""
    ids = np.concatenate(list(ids_parts), axis=1).astype(np.uint32)
    d = np.concatenate(list(dists_parts), axis=1).astype(np.float32)
    out_i = np.full((ids.shape[0], k), UINT32_MAX, np.uint32)
    out_d = np.full((ids.shape[0], k), np.inf, np.float32)
    for q in range(ids.shape[0]):
        live = ids[q] != UINT32_MAX
        li, ld = ids[q][live], d[q][live]
        order = np.lexsort((li, ld))[:k]
        out_i[q, :order.shape[0]] = li[order]
        out_d[q, :order.shape[0]] = ld[order]
    return out_i, out_d


class ShardedIndex:
    """One rank's share of a list-sharded index (see module docstring)."""

    def __init__(self, dim: int, nbits: int, seed: int = 0, group=None, make_engine=None, device: int | None = None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.dim, self.nbits, self.seed = dim, nbits, seed
        if make_engine is None:
            import e8qlib

            dev = self.rank if device is None else device
            make_engine = lambda: e8qlib.E8qIndex(dim, nbits, seed, device=dev)  # noqa: E731
        self.engine = make_engine()
        self.owner = None
        self.global_ids = None

    def build(self, data, centroids, cluster_ids):
        """Every rank passes the full data; each keeps the rows of its lists."""
        data = np.ascontiguousarray(data, np.float32)
        cluster_ids = np.ascontiguousarray(cluster_ids, np.uint32)
        nlist = np.asarray(centroids).shape[0]
        self.owner = partition_lists(np.bincount(cluster_ids, minlength=nlist), self.world)
        mine = np.nonzero(self.owner[cluster_ids] == self.rank)[0]
        self.global_ids = mine.astype(np.uint32)
        self.engine.build(data[mine], np.ascontiguousarray(centroids, np.float32), cluster_ids[mine])

    def search(self, queries, k: int, nprobe: int, **kw):
        """Local top-k over the owned lists, all-gather, merge; every rank
        returns the global (ids, dists)."""
        import torch

        ids, d = self.engine.search(queries, k, nprobe, **kw)
        ids = np.asarray(ids, np.uint32)
        live = ids != UINT32_MAX
        gids = np.full_like(ids, UINT32_MAX)
        gids[live] = self.global_ids[ids[live]]
        backend = self.dist.get_backend(self.group)
        dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
        ti = torch.from_numpy(gids.view(np.int32)).to(dev)
        td = torch.from_numpy(np.ascontiguousarray(d, np.float32)).to(dev)
        all_i = [torch.empty_like(ti) for _ in range(self.world)]
        all_d = [torch.empty_like(td) for _ in range(self.world)]
        self.dist.all_gather(all_i, ti, group=self.group)
        self.dist.all_gather(all_d, td, group=self.group)
        return merge_topk([t.cpu().numpy().view(np.uint32) for t in all_i], [t.cpu().numpy() for t in all_d], k)
