"""tcgen05 kind::i8 tensor-core contraction (the precision path's core)
against an integer reference."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,k", [(16, 32), (128, 64), (256, 256), (48, 96)])
def test_tc_i8_gemm_exact(n, k):
    import e8qlib._e8qlib as m

    rng = np.random.default_rng(n * 1000 + k)
    A = rng.integers(-128, 128, (128, k), dtype=np.int64).astype(np.int8)
    B = rng.integers(-128, 128, (n, k), dtype=np.int64).astype(np.int8)
    C, ms = m.tc_i8_gemm(A, B)
    ref = A.astype(np.int64) @ B.astype(np.int64).T
    assert np.array_equal(C.astype(np.int64), ref)
