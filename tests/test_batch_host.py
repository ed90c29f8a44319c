"""Host-side pieces of the batched driver that need no GPU: the scoped cap on
the host BLAS thread pools (numpy's and scipy's OpenBLAS)."""
import numpy as np
import scipy.linalg  # noqa: F401  (loads scipy's own OpenBLAS pool)
from threadpoolctl import threadpool_info

from rest_b200.scf_batch import host_blas_limit


def _blas_threads():
    return sorted(d["num_threads"] for d in threadpool_info() if d["user_api"] == "blas")


def test_blas_pools_are_capped_inside_and_restored_after():
    before = _blas_threads()
    with host_blas_limit(1):
        assert _blas_threads() == [1] * len(before)
        a = np.random.default_rng(0).standard_normal((64, 64))
        assert np.allclose(a @ np.linalg.inv(a), np.eye(64), atol=1e-8)
    assert _blas_threads() == before


def test_none_leaves_the_pools_alone():
    before = _blas_threads()
    with host_blas_limit(None):
        assert _blas_threads() == before


def test_pool_reuse_stays_within_the_budget():
    from rest_b200.scf_batch import pool_reuse

    # first group: nothing pooled yet
    assert pool_reuse([], [5.0, 4.0], 10.0) == 0
    # a smaller, equally long group fits in what the pool holds
    assert pool_reuse([5.0, 5.0], [3.0, 2.0], 10.0) == 2
    # a longer group: 2 reused (holding 5 each) + 2 fresh of 3 = 16 > 12 -> start afresh
    assert pool_reuse([5.0, 5.0], [3.0, 3.0, 3.0, 3.0], 12.0) == 0
    # ... and within a larger budget the pool is kept
    assert pool_reuse([5.0, 5.0], [3.0, 3.0, 3.0, 3.0], 16.0) == 2
    # a shorter group keeps only as many contexts as it has molecules
    assert pool_reuse([5.0, 5.0, 5.0], [4.0], 10.0) == 1
    # a molecule larger than what its context held counts at its own size
    assert pool_reuse([2.0, 2.0], [6.0, 1.0], 7.0) == 0
