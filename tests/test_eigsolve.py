"""Warm-started eigensolver (rest_b200.eigsolve.refine) on CPU: clustered
spectra in a padded batch, rejection of a basis that is too far off, and the
orthogonalised Fock matrices of a real SCF run ((H2O)2, def2-SVP, the SCF loop
of rest_b200.scf on the CPU oracle) refined from one iteration to the next."""
import numpy as np
import pytest
import torch

from rest_b200.eigsolve import refine


def _clustered(n, rng):
    """A spectrum like a water cluster's: tight groups (core, valence) and a spread."""
    groups = [-20.5 + 1e-3 * rng.standard_normal(4), -1.3 + 2e-3 * rng.standard_normal(4),
              -0.6 + 5e-3 * rng.standard_normal(4)]
    rest = np.sort(rng.uniform(0.1, 4.0, n - 12))
    return np.sort(np.concatenate(groups + [rest]))


def _batch(nv, nm, pert, seed=0):
    rng = np.random.default_rng(seed)
    B = len(nv)
    A = np.zeros((B, nm, nm))
    V0 = np.zeros((B, nm, nm))
    for b, n in enumerate(nv):
        w = _clustered(n, rng)
        Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
        M = (Q * w) @ Q.T
        P = rng.standard_normal((n, n))
        A[b, :n, :n] = M + pert * (P + P.T)
        V0[b, :n, :n] = Q  # eigenvectors of the unperturbed matrix
        A[b, n:, n:] = 1e6 * np.eye(nm - n)
        V0[b, n:, n:] = np.eye(nm - n)
    return torch.tensor(A), torch.tensor(V0)


def test_padded_batch_converges_to_eigh():
    nv, nm = [40, 33, 40, 27], 40
    A, V0 = _batch(nv, nm, 2e-3)
    lam, V, ok, off = refine(A, V0, nv, steps=9)
    assert bool(ok.all())
    for b, n in enumerate(nv):
        ref = np.linalg.eigvalsh(A[b, :n, :n].numpy())
        assert np.abs(lam[b, :n].numpy() - ref).max() < 1e-12
        Vb = V[b].numpy()
        assert np.abs(Vb.T @ Vb - np.eye(nm)).max() < 1e-13
        Sb = Vb[:n, :n].T @ A[b, :n, :n].numpy() @ Vb[:n, :n]
        assert np.abs(Sb - np.diag(np.diag(Sb))).max() < 1e-11
        # the padding stays the identity, eigenvalues 1e6 last
        assert np.array_equal(Vb[n:, n:], np.eye(nm - n)) and not Vb[:n, n:].any() and not Vb[n:, :n].any()
        assert np.all(lam[b, n:].numpy() == 1e6)


def test_basis_too_far_off_is_rejected():
    nv, nm = [30, 30], 30
    A, _ = _batch(nv, nm, 0.0)
    rng = np.random.default_rng(1)
    V0 = torch.tensor(np.stack([np.linalg.qr(rng.standard_normal((nm, nm)))[0] for _ in nv]))
    lam, V, ok, off = refine(A, V0, nv, steps=4)
    assert not bool(ok.any())


def test_eigenvalues_come_back_sorted_after_a_crossing():
    """Two levels that swap order between iterations: the refined pairs are re-sorted."""
    n = 6
    w0 = np.array([-2.0, -1.0, -0.50, -0.49, 1.0, 2.0])
    w1 = np.array([-2.0, -1.0, -0.48, -0.51, 1.0, 2.0])  # levels 2 and 3 cross
    Q, _ = np.linalg.qr(np.random.default_rng(2).standard_normal((n, n)))
    A = torch.tensor(((Q * w1) @ Q.T)[None])
    lam, V, ok, _ = refine(A, torch.tensor(Q[None]), [n], steps=3)
    assert bool(ok[0])
    assert np.allclose(lam[0].numpy(), np.sort(w1), atol=1e-14, rtol=0)


@pytest.fixture(scope="module")
def water_dimer_fock_sequence():
    from oracle.scf_ctx import OracleRIJK
    from rest_b200.geometry import water_cluster
    from rest_b200.scf import SCF, ScfOptions, _full

    seq = []

    class Recording(SCF):
        def diagonalize(self, fock_upper):
            seq.append(_full(fock_upper[0], self.n))
            return super().diagonalize(fock_upper)

    opts = ScfOptions(scf_acc_etot=1e-10, scf_acc_rho=1e-7, scf_acc_eev=1e-7, max_scf_cycle=60)
    s = Recording(water_cluster(2, seed=3), "def2-SVP", "def2-SVP-JKFIT", opts, ctx=OracleRIJK())
    assert s.run().converged
    w, u = np.linalg.eigh(s.ovlp)
    X = (u / np.sqrt(w)) @ u.T
    return [X @ F @ X for F in seq]


def test_refinement_along_a_water_dimer_scf(water_dimer_fock_sequence):
    """From the previous iteration's eigenvectors: every step whose Fock change is
    below 0.1 Eh passes within 4 + 5 steps with eigenvalues and occupied projector
    equal to LAPACK's; a step that does not pass is reported, never wrong."""
    seq = water_dimer_fock_sequence
    n, nocc = seq[0].shape[0], 10
    passed = 0
    for k in range(1, len(seq)):
        _, v0 = np.linalg.eigh(seq[k - 1])
        e1, v1 = np.linalg.eigh(seq[k])
        A = torch.tensor(seq[k])[None]
        lam, V, ok, off = refine(A, torch.tensor(v0)[None], [n], steps=4)
        if not bool(ok[0]) and float(off[0]) < 1e-2:
            lam, V, ok, off = refine(A, V, [n], steps=5)
        if np.abs(seq[k] - seq[k - 1]).max() < 0.1:
            assert bool(ok[0]), k
        if bool(ok[0]):
            passed += 1
            assert np.abs(lam[0].numpy() - e1).max() < 1e-12
            Vo = V[0].numpy()[:, :nocc]
            assert np.abs(Vo @ Vo.T - v1[:, :nocc] @ v1[:, :nocc].T).max() < 1e-12
    assert passed >= len(seq) // 2
