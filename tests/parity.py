"""Shared parity assertions for top-k results (test helper)."""
import numpy as np

RTOL = 1e-4  # plain-scan distances vs the reference's scalar estimator


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-3)


def assert_topk_parity(ids, dists, ref_ids, ref_dists, rtol=RTOL):
    """Distances within rtol of the reference position by position, the same
    padding (UINT32_MAX / +inf), and identical ids outside ties: any id that
    differs must sit at a distance within rtol of the reference's at that rank,
    and every reference id clearly inside the k-th distance must be present."""
    ids = np.asarray(ids)
    ref_ids = np.asarray(ref_ids)
    dists = np.asarray(dists, np.float32)
    ref_dists = np.asarray(ref_dists, np.float32)
    assert ids.shape == ref_ids.shape
    fin = np.isfinite(ref_dists)
    assert np.array_equal(np.isfinite(dists), fin), "padding differs"
    assert np.all(ids[~fin] == 0xFFFFFFFF)
    if fin.any():
        err = rel_err(dists[fin], ref_dists[fin])
        assert err.max() < rtol, f"max rel dist err {err.max():.3g}"
    for i in range(ids.shape[0]):
        row_fin = fin[i]
        if not row_fin.any():
            continue
        kth = ref_dists[i][row_fin].max()
        inside = ref_ids[i][row_fin & (ref_dists[i] < kth - rtol * max(abs(kth), 1e-3) * 2)]
        missing = set(inside.tolist()) - set(ids[i].tolist())
        assert not missing, f"row {i}: ids {sorted(missing)} missing outside ties"
        for j in np.nonzero(ids[i] != ref_ids[i])[0]:
            assert rel_err(dists[i, j], ref_dists[i, j]) < rtol
