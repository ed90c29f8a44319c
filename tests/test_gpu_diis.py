"""Batched DIIS coefficients on the device (rijk_diis_coefficients_dev) against
REST's diis_solver restated with NumPy (scf_io/mod.rs:3138-3188: the row sums of
B^-1 over their total; failure where the inverse does not exist)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rest_diis(gram, k):
    """REST's diis_solver on the leading k x k block: None when _dinverse fails."""
    try:
        binv = np.linalg.inv(gram[:k, :k])
    except np.linalg.LinAlgError:
        return None
    if not np.all(np.isfinite(binv)):
        return None
    return binv.sum(axis=0) / binv.sum()


def _run(grams, counts):
    import torch

    from rest_b200.eigsolve import diis_coefficients

    coef, failed = diis_coefficients(torch.as_tensor(grams, device="cuda"), counts)
    torch.cuda.synchronize()
    return coef.cpu().numpy(), failed.cpu().numpy()


def test_coefficients_match_rest_over_a_batch():
    rng = np.random.default_rng(5)
    B, m, L = 37, 8, 300
    grams = np.zeros((B, m, m))
    counts = []
    for b in range(B):
        k = 1 + b % m if b < 30 else m + 3 + b  # counts beyond m use all m slots
        kk = min(k, m)
        e = rng.standard_normal((kk, L)) * np.logspace(0, -2, kk)[:, None]  # shrinking errors, as in an SCF
        grams[b, :kk, :kk] = e @ e.T
        counts.append(k)
    coef, failed = _run(grams, counts)
    assert not failed.any()
    for b in range(B):
        kk = min(counts[b], m)
        ref = _rest_diis(grams[b], kk)
        assert np.allclose(coef[b, :kk], ref, rtol=1e-9, atol=1e-12)
        assert abs(coef[b, :kk].sum() - 1.0) < 1e-12
        assert np.all(coef[b, kk:] == 0.0)


def test_singular_and_empty_histories():
    m = 4
    grams = np.zeros((4, m, m))
    grams[0, :2, :2] = [[2.0, 2.0], [2.0, 2.0]]  # two identical error vectors: exactly singular
    grams[1, :3, :3] = np.diag([1.0, 2.0, 3.0])
    grams[2, :2, :2] = [[1.0, np.nan], [np.nan, 1.0]]
    counts = [2, 3, 2, 0]
    coef, failed = _run(grams, counts)
    assert _rest_diis(grams[0], 2) is None
    assert failed.tolist() == [True, False, True, False]
    assert coef[0].tolist() == [1.0, 0.0, 0.0, 0.0]
    assert coef[2].tolist() == [1.0, 0.0, 0.0, 0.0]
    assert np.allclose(coef[1, :3], _rest_diis(grams[1], 3), rtol=1e-14)
    assert coef[3].tolist() == [0.0] * m


def test_history_longer_than_the_kernel_limit_is_refused():
    import torch

    from rest_b200 import RijkError
    from rest_b200.eigsolve import diis_coefficients

    with pytest.raises(RijkError):
        diis_coefficients(torch.zeros(1, 33, 33, dtype=torch.float64, device="cuda"), [1])
