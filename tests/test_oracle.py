"""CPU checks of the FP64 oracle (no GPU): internal consistency of the
restated REST formulas and agreement with the committed golden fixtures."""
import numpy as np
import pytest

from oracle import rijk_oracle as O
from rest_b200.synth import host_case


def _spd(naux, seed, eps=1e-3):
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((naux, naux + 3))
    return np.asfortranarray(g @ g.T / naux + eps * np.eye(naux))


@pytest.mark.parametrize("n,naux", [(1, 3), (5, 20), (13, 40)])
def test_ri3fn_and_rimatr_forms_agree(n, naux):
    case = host_case(n, naux, max(1, n // 3), seed=n)
    ri3 = O.ri3fn_from_rimatr(case.rimatr, n)
    assert np.array_equal(O.rimatr_from_ri3fn(ri3), case.rimatr)
    dm = [case.dm, case.dm]
    a = O.vj_upper_with_ri_v(ri3, dm, 1, 1.0)[0]
    b = O.vj_upper_with_rimatr_v(case.rimatr, dm, 1, 1.0)[0]
    assert np.max(np.abs(a - b)) < 1e-12
    k1 = O.vk_upper_with_ri_v_use_dm_only(ri3, dm, 1, -0.5)[0]
    k2 = O.vk_upper_with_rimatr_use_dm_only(case.rimatr, dm, 1, -0.5)[0]
    assert np.max(np.abs(k1 - k2)) < 1e-12
    # occ form with D = C C^T equals the dm form
    homo = [case.nocc - 1, 0]
    occ = [np.ones(case.nocc), np.ones(1)]
    k3 = O.vk_upper_with_ri_v(ri3, [case.c_occ, case.c_occ], homo, occ, 1, -0.5)[0]
    assert np.max(np.abs(k1 - k3)) < 1e-12
    # full forms: upper part equals the packed result
    jf = O.vj_full_with_ri_v(ri3, dm, 1, 1.0)[0]
    assert np.max(np.abs(O.to_upper(jf) - a)) < 1e-12
    kf = O.vk_full_fromdm_with_ri_v(ri3, dm, 1, -0.5)[0]
    assert np.max(np.abs(O.to_upper(kf) - k1)) < 1e-12


def test_exchange_is_negative_semidefinite_and_symmetric():
    case = host_case(11, 44, 3, seed=7)
    ri3 = O.ri3fn_from_rimatr(case.rimatr, 11)
    kf = O.vk_full_fromdm_with_ri_v(ri3, [case.dm], 1, -1.0)[0]
    assert np.max(np.abs(kf - kf.T)) < 1e-13
    assert np.trace(case.dm @ kf) <= 1e-12


def test_metric_factors_give_the_same_fock_matrices():
    """REST's V^-1/2 and the Cholesky L^-T fit give identical J and K."""
    n, naux = 9, 30
    case = host_case(n, naux, 2, seed=3)
    v = _spd(naux, 5)
    int3c = case.rimatr  # any three-centre array works for the identity
    b_half = O.fit_rimatr(int3c, O.metric_inv_sqrt(v, 0.0))
    b_chol = O.fit_rimatr(int3c, O.metric_cholesky_inv_t(v))
    b_trsm = O.fit_rimatr_cholesky(int3c, v)
    assert np.max(np.abs(b_chol - b_trsm)) < 1e-10
    dm = [case.dm]
    for b in (b_chol, b_trsm):
        ja = O.vj_upper_with_rimatr_v(b_half, dm, 1, 1.0)[0]
        jb = O.vj_upper_with_rimatr_v(b, dm, 1, 1.0)[0]
        assert np.max(np.abs(ja - jb)) < 1e-9
        ka = O.vk_upper_with_rimatr_use_dm_only(b_half, dm, 1, -0.5)[0]
        kb = O.vk_upper_with_rimatr_use_dm_only(b, dm, 1, -0.5)[0]
        assert np.max(np.abs(ka - kb)) < 1e-9


def test_metric_threshold_drops_small_eigenvalues():
    naux = 12
    rng = np.random.default_rng(1)
    u = np.linalg.qr(rng.standard_normal((naux, naux)))[0]
    lam = np.logspace(-12, 0, naux)
    v = (u * lam) @ u.T
    m = O.metric_inv_sqrt(v)
    kept = lam >= O.AUXBAS_THRESHOLD
    assert np.linalg.matrix_rank(m, tol=1e-6) == kept.sum()
    with pytest.raises(np.linalg.LinAlgError):
        O.metric_cholesky_factor(v - 1e-3 * np.eye(naux))


def test_energy_contraction_matches_full_trace():
    rng = np.random.default_rng(0)
    a = rng.standard_normal((7, 7))
    a = a + a.T
    b = rng.standard_normal((7, 7))
    b = b + b.T
    e = O.par_energy_contraction(O.to_upper(a), O.to_upper(b))
    assert abs(e - 0.5 * np.sum(a * b)) < 1e-12


def test_occupation_and_density():
    occ, homo, lumo = O.occupation_integer(6, 5.0, 2.0)
    assert homo == 4 and lumo == 5 and occ.tolist() == [2, 2, 2, 2, 2, 0]
    occ, homo, _ = O.occupation_integer(6, 2.5, 1.0)
    assert homo == 2 and occ[2] == 0.5
    rng = np.random.default_rng(2)
    c = rng.standard_normal((6, 6))
    d = O.density_matrix(c, np.array([2.0, 2.0, 0, 0, 0, 0]), 1)
    assert np.allclose(d, 2.0 * c[:, :2] @ c[:, :2].T)
