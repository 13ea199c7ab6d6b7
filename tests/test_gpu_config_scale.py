"""Correctness at the headline configuration's scale (1M x 960-d mixture,
1,024 lists, nbits 6, k = 10, nprobe 64), where the C oracle is too slow to
run: properties that do not depend on size.

  * the plain, batched and precision paths return the same top-k (ids equal
    outside ties, distances within 1e-4), and the pruned path the same rows
    wherever its bound held (nearly all);
  * every returned distance is the estimator of its id (E8qIndex.estimate,
    one vector at a time) within 1e-5 relative;
  * rows are sorted by (distance, id) with unique ids;
  * recall@10 against FP64 brute force is at least 0.97.
"""
import numpy as np
import pytest

from parity import assert_topk_parity

pytestmark = pytest.mark.gpu


class _Cfg:
    n, dim, nlist, seed, pool = 1_000_000, 960, 1024, 0, 256
    spectrum, sigma = 0.5, 0.4


@pytest.fixture(scope="module")
def scale():
    import torch

    import bench as B
    import e8qlib

    dev = torch.device("cuda", 0)
    x, cm, lab, q = B.gen_data(_Cfg, dev, 0)
    sp = torch.cuda.current_stream().cuda_stream
    idx = e8qlib.E8qIndex(_Cfg.dim, 6, 0, device=0)
    idx.build_ptr(x.data_ptr(), _Cfg.n, cm.data_ptr(), _Cfg.nlist, lab.data_ptr(), 0.0, sp)
    torch.cuda.synchronize()
    gt = B.ground_truth(x, q[:64], 10)
    qn = q[:64].cpu().numpy()
    yield idx, qn, gt, B
    del idx, x, cm, lab, q
    torch.cuda.empty_cache()


def test_paths_agree_at_config_scale(scale):
    idx, qn, gt, B = scale
    pi, pd = idx.search(qn, 10, 64, mode="plain")
    for mode in ("batched", "precision"):
        ids, d = idx.search(qn, 10, 64, mode=mode)
        assert_topk_parity(ids, d, pi, pd)
    ids, d = idx.search(qn, 10, 64, mode="pruned")
    same_rows = np.mean([np.array_equal(a, b) for a, b in zip(ids, pi)])
    assert same_rows >= 0.95, same_rows


def test_rows_are_the_estimator_sorted_and_unique(scale):
    idx, qn, gt, B = scale
    ids, d = idx.search(qn, 10, 64, mode="plain")
    for r in range(len(ids)):
        assert len(set(ids[r].tolist())) == ids.shape[1]
        key = list(zip(d[r].tolist(), ids[r].tolist()))
        assert key == sorted(key)
    rng = np.random.default_rng(5)
    for r in rng.choice(len(ids), 8, replace=False):
        for j in (0, 4, 9):
            est = idx.estimate(qn[r], int(ids[r, j]))
            assert abs(est - d[r, j]) <= 1e-5 * max(1.0, abs(d[r, j]))


def test_recall_against_fp64_at_config_scale(scale):
    idx, qn, gt, B = scale
    ids, _ = idx.search(qn, 10, 64, mode="plain")
    assert B.recall_at(ids, gt, 10) >= 0.97
