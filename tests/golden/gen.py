"""Deterministic, platform-exact test inputs for the golden fixtures.

Values are sums of 16-bit integer hashes scaled by a power of two, so every
float32 is produced by exact integer arithmetic: the same bits on any machine
and any numpy version. The golden fixtures store only outputs; the tests
regenerate the inputs from these functions.
"""
from __future__ import annotations

import numpy as np

_M = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def det_u64(seed: int, n: int) -> np.ndarray:
    idx = np.arange(n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        return _splitmix(idx * np.uint64(0x632BE59BD9B4E019) + np.uint64(seed & 0xFFFFFFFF) *
                         np.uint64(0x9E3779B97F4A7C15) + np.uint64(1))


def det_normal(seed: int, shape) -> np.ndarray:
    """Approximately N(0,1) (Irwin-Hall of four 16-bit uniforms), exact float32."""
    n = int(np.prod(shape))
    h = det_u64(seed, n)
    s = np.zeros(n, np.int64)
    for j in range(4):
        s += ((h >> np.uint64(16 * j)) & np.uint64(0xFFFF)).astype(np.int64)
    # mean 4*32767.5, sd sqrt(4*(65536^2-1)/12) ~ 37837; scale by 2^-15 ~ 0.87 sd
    v = (s - 131070).astype(np.float64) / 32768.0
    return v.astype(np.float32).reshape(shape)


def det_int(seed: int, n: int, hi: int) -> np.ndarray:
    return (det_u64(seed, n) % np.uint64(hi)).astype(np.uint32)


def det_unit(seed: int, n: int, dim: int) -> np.ndarray:
    x = det_normal(seed, (n, dim)).astype(np.float64)
    x /= np.sqrt((x * x).sum(axis=1, keepdims=True))
    return x.astype(np.float32)


def det_mixture(seed: int, n: int, dim: int, nlist: int, sigma: float = 0.5):
    """Gaussian-mixture-like base: centres + sigma * noise, labels = component,
    centroids = per-component means (float64 mean cast to float32)."""
    cen = det_normal(seed * 3 + 1, (nlist, dim))
    lab = det_int(seed * 3 + 2, n, nlist)
    x = (cen[lab] + np.float32(sigma) * det_normal(seed * 3 + 3, (n, dim))).astype(np.float32)
    cm = np.zeros((nlist, dim), np.float32)
    for c in range(nlist):
        m = lab == c
        cm[c] = x[m].astype(np.float64).mean(0) if m.any() else cen[c]
    return x, cm, lab
