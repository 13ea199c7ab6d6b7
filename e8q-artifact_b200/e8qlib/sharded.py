"""List-sharded IVF search across GPUs: one process per GPU, IVF lists
partitioned over the ranks, one exchange step.

Lists are independent, so each rank holds the vectors of the lists it owns
(all centroids are replicated, so every rank routes a query to the same
probes; lists it does not own are empty locally) and scans only those. The
one collective is an all-gather of every rank's local top-k (distance, id)
per query; the merge keeps the k best under the reference's total order --
smaller distance first, ties by smaller id (src/index/e8q_internal.hpp:47-49),
padding (UINT32_MAX, +inf) last. With the NCCL backend the rows stay on the
GPU: the local results are gathered device to device and merged there with
one sort of 64-bit (distance, id) keys per query; with gloo the same keys are
sorted on the host.

E8Q: each rank centres its own vectors on their own mean; the estimator's
residual to the list centroid does not depend on that mean, so sharded
distances match a single index's up to float rounding. ME8Q: the bit plan
follows the per-dimension variance, so every rank must build with the same
``variance`` (the whole data's); ``ShardedIndex.build`` passes it through.
The merge equals one index's result for the exact modes (``mode="batched"``
or ``"plain"``). The pruned modes (both engines' default, as in the
reference) prune against each rank's own running top-k, so a sharded pruned
search can keep rows a single index's cascade would have cut, and the
reverse where the bound fails; pass ``mode="batched"`` for the single index's
exact rows.

The per-rank engine is any object with ``build(data, centroids, cluster_ids,
**kw)`` and ``search(queries, k, nprobe, **kw) -> (ids, dists)``; by default an
``e8qlib.E8qIndex`` (``kind="e8q"``) or ``e8qlib.Me8qIndex``
(``kind="me8q"``) on this rank's GPU.
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


def _order_keys_np(ids, d):
    """int64 keys whose order is (distance, id): the float's bits mapped to a
    signed integer of the same order (-0 taken as +0), then the id."""
    d = np.ascontiguousarray(d, np.float32) + np.float32(0.0)
    b = d.view(np.int32).astype(np.int64)
    b = np.where(b < 0, b ^ 0x7FFFFFFF, b)
    return (b << 32) | ids.astype(np.int64)


def merge_topk(ids_parts, dists_parts, k: int):
    """Merge per-rank top-k rows ([world, nq, k] each) into the global top-k
    under (distance, id) order; padding entries sort last."""
    ids = np.concatenate(list(ids_parts), axis=1).astype(np.uint32)
    d = np.concatenate(list(dists_parts), axis=1).astype(np.float32)
    key = _order_keys_np(ids, d)
    order = np.argsort(key, axis=1, kind="stable")[:, :k]
    out_i = np.take_along_axis(ids, order, 1)
    out_d = np.take_along_axis(d, order, 1)
    if out_i.shape[1] < k:
        pad = k - out_i.shape[1]
        out_i = np.concatenate([out_i, np.full((ids.shape[0], pad), UINT32_MAX, np.uint32)], 1)
        out_d = np.concatenate([out_d, np.full((ids.shape[0], pad), np.inf, np.float32)], 1)
    return out_i, out_d


def merge_topk_torch(ids, d, k: int):
    """The same merge on the device: ids (int32 holding uint32) and d of shape
    [nq, m], one ascending sort of the 64-bit keys per row."""
    import torch

    d = d.float() + 0.0
    b = d.view(torch.int32).to(torch.int64)
    b = torch.where(b < 0, b ^ 0x7FFFFFFF, b)
    key = (b << 32) | (ids.to(torch.int64) & 0xFFFFFFFF)
    sk, order = torch.sort(key, dim=1, stable=True)
    order = order[:, :k]
    return torch.gather(ids, 1, order), torch.gather(d, 1, order)


class ShardedIndex:
    """One rank's share of a list-sharded index (see module docstring)."""

    def __init__(self, dim: int, nbits: float = 4, seed: int = 0, group=None, make_engine=None,
                 device: int | None = None, kind: str = "e8q"):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.dim, self.nbits, self.seed = dim, nbits, seed
        if make_engine is None:
            import e8qlib

            dev = self.rank if device is None else device
            if kind == "e8q":
                make_engine = lambda: e8qlib.E8qIndex(dim, int(nbits), seed, device=dev)  # noqa: E731
            elif kind == "me8q":
                make_engine = lambda: e8qlib.Me8qIndex(dim, float(nbits), seed, device=dev)  # noqa: E731
            else:
                raise ValueError("kind must be 'e8q' or 'me8q'")
        self.engine = make_engine()
        self.owner = None
        self.global_ids = None

    def build(self, data, centroids, cluster_ids, **kw):
        """Every rank passes the full data; each keeps the rows of its lists.
        Keyword arguments go to every rank's engine (ME8Q: pass the whole
        data's ``variance`` so all ranks use one bit plan)."""
        data = np.ascontiguousarray(data, np.float32)
        cluster_ids = np.ascontiguousarray(cluster_ids, np.uint32)
        nlist = np.asarray(centroids).shape[0]
        self.owner = partition_lists(np.bincount(cluster_ids, minlength=nlist), self.world)
        mine = np.nonzero(self.owner[cluster_ids] == self.rank)[0]
        self.global_ids = mine.astype(np.uint32)
        self.engine.build(data[mine], np.ascontiguousarray(centroids, np.float32), cluster_ids[mine], **kw)

    def search(self, queries, k: int, nprobe: int, **kw):
        """Local top-k over the owned lists, all-gather, merge; every rank
        returns the global (ids, dists) as numpy arrays."""
        import torch

        ids, d = self.engine.search(queries, k, nprobe, **kw)
        ids = np.asarray(ids, np.uint32)
        live = ids != UINT32_MAX
        gids = np.full_like(ids, UINT32_MAX)
        gids[live] = self.global_ids[ids[live]]
        backend = self.dist.get_backend(self.group)
        if backend == "nccl":
            dev = torch.device("cuda", torch.cuda.current_device())
            ti = torch.from_numpy(gids.view(np.int32)).to(dev)
            td = torch.from_numpy(np.ascontiguousarray(d, np.float32)).to(dev)
            all_i = torch.empty((self.world,) + tuple(ti.shape), dtype=ti.dtype, device=dev)
            all_d = torch.empty((self.world,) + tuple(td.shape), dtype=td.dtype, device=dev)
            self.dist.all_gather_into_tensor(all_i, ti, group=self.group)
            self.dist.all_gather_into_tensor(all_d, td, group=self.group)
            nq = ti.shape[0]
            mi, md = merge_topk_torch(all_i.permute(1, 0, 2).reshape(nq, -1),
                                      all_d.permute(1, 0, 2).reshape(nq, -1), k)
            return mi.cpu().numpy().view(np.uint32), md.cpu().numpy()
        ti = torch.from_numpy(gids.view(np.int32))
        td = torch.from_numpy(np.ascontiguousarray(d, np.float32))
        all_i = [torch.empty_like(ti) for _ in range(self.world)]
        all_d = [torch.empty_like(td) for _ in range(self.world)]
        self.dist.all_gather(all_i, ti, group=self.group)
        self.dist.all_gather(all_d, td, group=self.group)
        return merge_topk([t.numpy().view(np.uint32) for t in all_i], [t.numpy() for t in all_d], k)
