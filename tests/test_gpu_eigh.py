"""The library's batched symmetric eigensolver (rijk_eigh_batched_dev) against
torch.linalg.eigh (cuSOLVER), FP64.

Random symmetric matrices, a matrix with exactly repeated eigenvalues, and the
orthogonalised Fock matrices of the batched SCF: eigenvalues within 1e-12 of
the largest in magnitude, residual |A v - lam v| and orthogonality |V^T V - I|
within 1e-12; padding keeps its pad value and unit vectors.
"""
import numpy as np
import pytest
import torch

from rest_b200.eigsolve import eigh_batched

pytestmark = pytest.mark.gpu


def _check(A, nvalid, lam, V, ok, tol=1e-12):
    assert bool(ok.all())
    for b, n in enumerate(nvalid):
        a = A[b, :n, :n]
        ref = torch.linalg.eigvalsh(a)
        scale = float(ref.abs().max()) if n else 1.0
        if n:
            assert float((lam[b, :n] - ref).abs().max()) <= tol * max(scale, 1.0)
        v = V[b, :n, :n]
        if n:
            assert float((a @ v - v * lam[b, :n][None, :]).abs().max()) <= tol * max(scale, 1.0) * 10
            assert float((v.T @ v - torch.eye(n, dtype=v.dtype, device=v.device)).abs().max()) <= tol * 10
        nm = A.shape[1]
        assert bool((lam[b, n:] == 1e6).all())
        pad = V[b, n:, n:]
        assert bool((pad == torch.eye(nm - n, dtype=v.dtype, device=v.device)).all())
        assert bool((V[b, :n, n:] == 0).all()) and bool((V[b, n:, :n] == 0).all())


@pytest.mark.parametrize("nm,nvalid", [(1, [1]), (7, [7, 2, 1, 5]), (100, [100, 37, 64, 3, 99]),
                                       (384, [384, 200]), (577, [577])])
def test_random_symmetric(nm, nvalid):
    rng = np.random.default_rng(nm)
    A = torch.zeros(len(nvalid), nm, nm, dtype=torch.float64, device="cuda")
    for b, n in enumerate(nvalid):
        m = rng.standard_normal((n, n))
        A[b, :n, :n] = torch.as_tensor(m + m.T, device="cuda")
    lam, V, ok = eigh_batched(A, nvalid)
    _check(A, nvalid, lam, V, ok)


def test_repeated_eigenvalues_and_diagonal_input():
    rng = np.random.default_rng(3)
    n = 60
    q = np.linalg.qr(rng.standard_normal((n, n)))[0]
    w = np.repeat([-2.0, 0.5, 3.0], 20)
    A = torch.stack([torch.as_tensor(q @ np.diag(w) @ q.T, device="cuda"),
                     torch.diag(torch.as_tensor(np.linspace(5, -5, n), device="cuda")),
                     torch.zeros(n, n, dtype=torch.float64, device="cuda")])
    lam, V, ok = eigh_batched(A, [n, n, n])
    _check(A, [n, n, n], lam, V, ok)


def test_orthogonalised_fock_matrices_of_water_clusters():
    """X^T F X of the first SCF iteration (hcore Fock) of uneven clusters."""
    from rest_b200.geometry import water_cluster
    from rest_b200.scf_batch import BatchedRHF

    mols = [water_cluster(k, seed=30 + k) for k in (1, 4, 2)]
    b = BatchedRHF(mols, "def2-SVP", "def2-SVP-JKFIT", precision="fp64", metric="cholesky")
    try:
        A = b.X.transpose(1, 2) @ b.H @ b.X
        A = 0.5 * (A + A.transpose(1, 2))
        lam, V, ok = eigh_batched(A, b.n)
        _check(A, b.n, lam, V, ok, tol=1e-11)
    finally:
        b.close()
