"""GPU parity of the RI J/K build against the FP64 oracle, through the C ABI.

Tolerance (the FP64 plain form's contract): max |GPU - oracle| <= 1e-10 per
element of every J/K matrix.
"""
import numpy as np
import pytest

from oracle import rijk_oracle as O
from rest_b200.synth import host_case

pytestmark = pytest.mark.gpu

TOL = 1e-10

SHAPES = [(1, 3, 1), (5, 17, 2), (7, 33, 3), (24, 113, 5), (33, 70, 4), (37, 150, 6), (100, 400, 16), (200, 800, 33)]


def _maxdiff(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))))


def _second_spin(case, seed):
    rng = np.random.default_rng(seed)
    c2 = np.asfortranarray(np.linalg.qr(rng.standard_normal((case.n, max(1, case.nocc - 1))))[0])
    return c2, np.asfortranarray(c2 @ c2.T)


@pytest.mark.parametrize("n,naux,nocc", SHAPES)
def test_vj_upper_rimatr_and_ri3fn(ctx, n, naux, nocc):
    case = host_case(n, naux, nocc, seed=100 + n)
    _, dm2 = _second_spin(case, n)
    ri3 = O.ri3fn_from_rimatr(case.rimatr, n)
    for spin in (1, 2):
        dm = [case.dm, dm2][:spin]
        ctx.set_rimatr(case.rimatr, n)
        got = ctx.vj_upper_with_rimatr_v(dm, spin, 1.0)
        ref = O.vj_upper_with_rimatr_v(case.rimatr, dm, spin, 1.0)
        for s in range(spin):
            assert _maxdiff(got[s], ref[s]) <= TOL
        ctx.set_ri3fn(ri3)
        got = ctx.vj_upper_with_ri_v(dm, spin, 0.5)
        ref = O.vj_upper_with_ri_v(ri3, dm, spin, 0.5)
        for s in range(spin):
            assert _maxdiff(got[s], ref[s]) <= TOL
        if spin == 1:
            assert got[1].shape == (1,)  # REST's placeholder slot


@pytest.mark.parametrize("n,naux,nocc", [(7, 33, 3), (37, 150, 6)])
def test_vj_modes_differ_exactly_as_rest_for_nonsymmetric_dm(ctx, n, naux, nocc):
    case = host_case(n, naux, nocc, seed=5)
    rng = np.random.default_rng(9)
    d = np.asfortranarray(rng.standard_normal((n, n)))
    ctx.set_rimatr(case.rimatr, n)
    ri3 = O.ri3fn_from_rimatr(case.rimatr, n)
    a = ctx.vj_upper_with_ri_v([d], 1, 1.0)[0]
    b = ctx.vj_upper_with_rimatr_v([d], 1, 1.0)[0]
    assert _maxdiff(a, O.vj_upper_with_ri_v(ri3, [d], 1, 1.0)[0]) <= TOL
    assert _maxdiff(b, O.vj_upper_with_rimatr_v(case.rimatr, [d], 1, 1.0)[0]) <= TOL
    assert _maxdiff(a, b) > 1e-6  # the two REST formulas disagree for non-symmetric D
    jf = ctx.vj_full_with_ri_v([d], 1, 2.0)[0]
    assert _maxdiff(jf, O.vj_full_with_ri_v(ri3, [d], 1, 2.0)[0]) <= TOL


@pytest.mark.parametrize("n,naux,nocc", SHAPES)
def test_vk_occupied_form(ctx, n, naux, nocc):
    case = host_case(n, naux, nocc, seed=200 + n)
    c2, _ = _second_spin(case, n + 1)
    ctx.set_rimatr(case.rimatr, n)
    ri3 = O.ri3fn_from_rimatr(case.rimatr, n)
    num_state = nocc + 2
    e1 = np.zeros((n, num_state), order="F")
    e1[:, :nocc] = case.c_occ
    e2 = np.zeros((n, num_state), order="F")
    e2[:, : c2.shape[1]] = c2
    occ1 = np.zeros(num_state)
    occ1[:nocc] = 2.0
    occ2 = np.zeros(num_state)
    occ2[: c2.shape[1]] = 1.0
    occ2[0] = 0.5
    for spin, scale in ((1, -0.5), (2, -1.0)):
        eig = [e1, e2][:spin]
        homo = [nocc - 1, c2.shape[1] - 1][:spin]
        occ = [occ1, occ2][:spin]
        got = ctx.vk_upper_with_ri_v(eig, homo, occ, spin, scale)
        ref = O.vk_upper_with_ri_v(ri3, eig, homo, occ, spin, scale)
        for s in range(spin):
            assert _maxdiff(got[s], ref[s]) <= TOL


@pytest.mark.parametrize("n,naux,nocc", SHAPES[:-1])
def test_vk_density_forms(ctx, n, naux, nocc):
    case = host_case(n, naux, nocc, seed=300 + n)
    _, dm2 = _second_spin(case, n + 2)
    ri3 = O.ri3fn_from_rimatr(case.rimatr, n)
    for spin in (1, 2):
        dm = [case.dm, dm2][:spin]
        ctx.set_ri3fn(ri3)
        got = ctx.vk_upper_with_ri_v_use_dm_only(dm, spin, -0.5)
        ref = O.vk_upper_with_ri_v_use_dm_only(ri3, dm, spin, -0.5)
        for s in range(spin):
            assert _maxdiff(got[s], ref[s]) <= TOL
        ctx.set_rimatr(case.rimatr, n)
        got = ctx.vk_upper_with_rimatr_use_dm_only(dm, spin, -1.0)
        ref = O.vk_upper_with_rimatr_use_dm_only(case.rimatr, dm, spin, -1.0)
        for s in range(spin):
            assert _maxdiff(got[s], ref[s]) <= TOL


@pytest.mark.parametrize("n,naux,nocc", [(5, 17, 2), (37, 150, 6), (130, 300, 8)])
def test_vk_full_from_nonsymmetric_dm(ctx, n, naux, nocc):
    case = host_case(n, naux, nocc, seed=400 + n)
    rng = np.random.default_rng(n)
    d = np.asfortranarray(rng.standard_normal((n, n)) / n)
    ctx.set_rimatr(case.rimatr, n)
    ri3 = O.ri3fn_from_rimatr(case.rimatr, n)
    got = ctx.vk_full_fromdm_with_ri_v([d], 1, 1.0)[0]
    ref = O.vk_full_fromdm_with_ri_v(ri3, [d], 1, 1.0)[0]
    assert _maxdiff(got, ref) <= TOL
    assert _maxdiff(got, got.T) > 1e-8  # non-symmetric D gives a non-symmetric K


@pytest.mark.parametrize("n,naux", [(1, 3), (33, 70), (200, 800)])
def test_tensor_round_trip_is_bit_exact(ctx, n, naux):
    case = host_case(n, naux, 1, seed=n)
    ctx.set_rimatr(case.rimatr, n)
    assert np.array_equal(ctx.get_rimatr(), case.rimatr)
    ctx.set_ri3fn(O.ri3fn_from_rimatr(case.rimatr, n))
    assert np.array_equal(ctx.get_rimatr(), case.rimatr)


def _spd(naux, seed, eps=1e-2):
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((naux, naux + 5))
    return np.asfortranarray(g @ g.T / naux + eps * np.eye(naux))


@pytest.mark.parametrize("n,naux", [(5, 17), (24, 113), (40, 330)])
def test_metric_cholesky_fit(ctx, n, naux):
    case = host_case(n, naux, 2, seed=600 + n)
    v = _spd(naux, naux)
    int3c = case.rimatr
    ctx.build_rimatr_cholesky(v, int3c, n)
    got = ctx.get_rimatr()
    ref = O.fit_rimatr_cholesky(int3c, v)
    scale = max(1.0, float(np.max(np.abs(ref))))
    assert _maxdiff(got, ref) <= 1e-11 * scale * naux
    # J/K from the device fit equal those from REST's V^-1/2 whitening
    b_half = O.fit_rimatr(int3c, O.metric_inv_sqrt(v))
    j_ref = O.vj_upper_with_rimatr_v(b_half, [case.dm], 1, 1.0)[0]
    j_got = ctx.vj_upper_with_rimatr_v([case.dm], 1, 1.0)[0]
    assert _maxdiff(j_got, j_ref) <= 1e-9 * max(1.0, float(np.max(np.abs(j_ref))))


def test_metric_factor_fit_matches_rest_whitening(ctx):
    n, naux = 24, 113
    case = host_case(n, naux, 5, seed=11)
    v = _spd(naux, 3)
    m = O.metric_inv_sqrt(v)
    ctx.fit_rimatr(m, case.rimatr, n)
    ref = O.fit_rimatr(case.rimatr, m)
    assert _maxdiff(ctx.get_rimatr(), ref) <= 1e-12 * naux * max(1.0, float(np.max(np.abs(ref))))


def test_non_spd_metric_reports_the_failing_pivot(ctx):
    from rest_b200 import RijkError

    n, naux = 5, 40
    case = host_case(n, naux, 2, seed=1)
    v = _spd(naux, 4)
    v[37, 37] = -5.0
    with pytest.raises(RijkError) as ei:
        ctx.build_rimatr_cholesky(v, case.rimatr, n)
    assert ei.value.status == 3
    assert ei.value.failed_pivot == 38
    # the context is still usable afterwards
    ctx.set_rimatr(case.rimatr, n)
    ctx.vj_upper_with_rimatr_v([case.dm], 1, 1.0)


def test_bad_arguments_are_rejected(ctx):
    from rest_b200 import RijkError

    case = host_case(7, 20, 2, seed=1)
    ctx.set_rimatr(case.rimatr, 7)
    with pytest.raises(RijkError) as ei:
        ctx.vj_upper_with_rimatr_v([case.dm, case.dm, case.dm], 3, 1.0)
    assert ei.value.status == 1
    e = np.zeros((7, 3), order="F")
    with pytest.raises(RijkError):
        ctx.vk_upper_with_ri_v([e], [5], [np.ones(3)], 1, 1.0)  # homo beyond num_state
    with pytest.raises(RijkError):
        ctx.vk_upper_with_ri_v([e], [1], [np.array([1.0, -1.0, 0.0])], 1, 1.0)  # negative occupation


def test_density_matrix(ctx):
    rng = np.random.default_rng(8)
    n = 45
    c = np.asfortranarray(rng.standard_normal((n, n)))
    occ, homo, _ = O.occupation_integer(n, 7.0, 2.0)
    got = ctx.density_matrix([c], [homo], [occ], 1)[0]
    assert _maxdiff(got, O.density_matrix(c, occ, homo)) <= TOL


def test_full_size_n600_against_oracle(ctx):
    """The middle sweep size end to end: host-drawn tensor, J and K vs the oracle."""
    n = 600
    case = host_case(n, seed=7)
    ctx.set_rimatr(case.rimatr, n)
    j = ctx.vj_upper_with_rimatr_v([case.dm], 1, 1.0)[0]
    assert _maxdiff(j, O.vj_upper_with_rimatr_v(case.rimatr, [case.dm], 1, 1.0)[0]) <= TOL
    occ = np.ones(case.nocc)
    k = ctx.vk_upper_with_ri_v([case.c_occ], [case.nocc - 1], [occ], 1, -1.0)[0]
    # oracle K in the occupied form straight from rimatr, P by P
    ii, jj = O.upper_pairs(n)
    kref = np.zeros((n, n))
    for p in range(case.naux):
        bp = np.zeros((n, n))
        bp[ii, jj] = case.rimatr[:, p]
        bp[jj, ii] = case.rimatr[:, p]
        x = bp @ case.c_occ
        kref += x @ x.T
    assert _maxdiff(k, -kref[ii, jj]) <= TOL


def test_full_size_n1200_properties(ctx):
    """Largest sweep size (28 GB tensor, device-drawn): size-independent identities."""
    import torch

    from rest_b200.synth import device_case

    n = 1200
    with torch.cuda.stream(torch.cuda.ExternalStream(ctx.stream)):
        _n1200_body(ctx, n)


def _n1200_body(ctx, n):
    import torch

    from rest_b200.synth import device_case

    c_cm, dm = device_case(ctx, n, seed=99)
    nocc = c_cm.shape[0]
    npair = n * (n + 1) // 2
    dev = c_cm.device
    st = torch.cuda.current_stream().cuda_stream
    occ = torch.ones(nocc, dtype=torch.float64, device=dev)
    k_occ = torch.empty(npair, dtype=torch.float64, device=dev)
    k_dm = torch.empty(npair, dtype=torch.float64, device=dev)
    ctx.vk_upper_occ_dev(c_cm.data_ptr(), nocc, [nocc - 1], occ.data_ptr(), 1, -1.0, k_occ.data_ptr(), st)
    ctx.vk_upper_dm_dev(dm.data_ptr(), 1, -1.0, k_dm.data_ptr(), st)
    # J is linear in D: J(2D) - 2 J(D) == 0, and <D, J(D)> = sum_P w_P^2 >= 0
    j1 = torch.empty(npair, dtype=torch.float64, device=dev)
    j2 = torch.empty(npair, dtype=torch.float64, device=dev)
    dm2 = (2.0 * dm).contiguous()
    ctx.vj_upper_dev(dm.data_ptr(), 1, 1.0, 1, j1.data_ptr(), st)
    ctx.vj_upper_dev(dm2.data_ptr(), 1, 1.0, 1, j2.data_ptr(), st)
    ctx.synchronize(st)
    torch.cuda.synchronize()
    # occupied-orbital K and density K are two independent kernel paths
    assert float((k_occ - k_dm).abs().max()) <= TOL
    assert float((j2 - 2.0 * j1).abs().max()) <= TOL
    # REST's packed order is (i <= j) sorted by j then i == tril_indices (r=j, c=i)
    il = torch.tril_indices(n, n, device=dev)
    d_up = dm[il[1], il[0]]
    diag = torch.arange(n, device=dev)
    dg = diag * (diag + 1) // 2 + diag
    e = 2.0 * torch.dot(d_up, j1) - torch.dot(d_up[dg], j1[dg])
    assert float(e) > 0
    ek = 2.0 * torch.dot(d_up, k_occ) - torch.dot(d_up[dg], k_occ[dg])
    assert float(ek) < 0


def test_autotuner_picks_a_shape_and_keeps_results(ctx):
    n, naux, nocc = 200, 800, 33
    case = host_case(n, naux, nocc, seed=77)
    ctx.set_rimatr(case.rimatr, n)
    try:
        bh, br, ms = ctx.autotune(nocc, 256)
        assert 0 <= bh <= 5 and 0 <= br <= 5 and len(ms) == 6
        assert all(v[0] > 0 and v[1] > 0 for v in ms.values())
        assert ms[bh][0] == min(v[0] for v in ms.values())
        occ = np.full(nocc, 2.0)
        ri3 = O.ri3fn_from_rimatr(case.rimatr, n)
        k = ctx.vk_upper_with_ri_v([case.c_occ], [nocc - 1], [occ], 1, -0.5)[0]
        assert _maxdiff(k, O.vk_upper_with_ri_v(ri3, [case.c_occ], [nocc - 1], [occ], 1, -0.5)[0]) <= TOL
    finally:
        ctx.set_tiles(1, 1)


@pytest.mark.parametrize("n,naux,rows,cols", [(7, 33, (2, 7), (0, 2)), (37, 150, (6, 37), (0, 6)),
                                              (130, 300, (20, 130), (3, 20))])
def test_ao2mo_ri3mo(ctx, n, naux, rows, cols):
    case = host_case(n, naux, 2, seed=900 + n)
    rng = np.random.default_rng(n)
    c = np.asfortranarray(rng.standard_normal((n, n)) / np.sqrt(n))
    ctx.set_rimatr(case.rimatr, n)
    got = ctx.ao2mo([c, c[:, ::-1]], range(*rows), range(*cols), spin_channel=2)
    for s, cs in enumerate([c, np.asfortranarray(c[:, ::-1])]):
        ref = O.ao2mo(case.rimatr, cs, range(*rows), range(*cols))
        assert got[s].shape == ref.shape
        assert _maxdiff(got[s], ref) <= TOL


@pytest.mark.parametrize("ht,rk", [(0, 0), (1, 1), (2, 2), (3, 3), (4, 4), (5, 5), (2, 1), (1, 3), (4, 1), (1, 4),
                                   (5, 1), (1, 5)])
def test_every_tile_shape_gives_the_same_k(ctx, ht, rk):
    n, naux, nocc = 150, 300, 40
    case = host_case(n, naux, nocc, seed=31)
    ri3 = O.ri3fn_from_rimatr(case.rimatr, n)
    ctx.set_rimatr(case.rimatr, n)
    try:
        ctx.set_tiles(ht, rk)
        occ = np.full(nocc, 2.0)
        k = ctx.vk_upper_with_ri_v([case.c_occ], [nocc - 1], [occ], 1, -0.5)[0]
        assert _maxdiff(k, O.vk_upper_with_ri_v(ri3, [case.c_occ], [nocc - 1], [occ], 1, -0.5)[0]) <= TOL
        kd = ctx.vk_upper_with_rimatr_use_dm_only([case.dm], 1, -1.0)[0]
        assert _maxdiff(kd, O.vk_upper_with_rimatr_use_dm_only(case.rimatr, [case.dm], 1, -1.0)[0]) <= TOL
        rng = np.random.default_rng(3)
        d = np.asfortranarray(rng.standard_normal((n, n)) / n)
        kf = ctx.vk_full_fromdm_with_ri_v([d], 1, 1.0)[0]
        assert _maxdiff(kf, O.vk_full_fromdm_with_ri_v(ri3, [d], 1, 1.0)[0]) <= TOL
    finally:
        ctx.set_tiles(1, 1)


def test_smaller_tensor_reuses_the_allocation(ctx):
    """A context keeps its tensor allocation when a smaller tensor replaces a
    larger one (the molecule-set driver reuses contexts, largest molecules
    first): results equal a fresh load's, and the reported size is the new
    tensor's."""
    big = host_case(100, 400, 16, seed=31)
    small = host_case(37, 150, 6, seed=32)
    ctx.set_rimatr(big.rimatr, 100)
    size_big = ctx.tensor_bytes()
    ctx.set_rimatr(small.rimatr, 37)
    size_small = ctx.tensor_bytes()
    assert 0 < size_small < size_big
    nt = -(-37 // 32)
    assert size_small == (-(-150 // 32) * 32) * nt * (nt + 1) // 2 * 1024 * 8
    assert np.array_equal(ctx.get_rimatr(), small.rimatr)
    eig = np.zeros((37, 8), order="F")
    eig[:, :6] = small.c_occ
    occ = [np.r_[np.full(6, 2.0), np.zeros(2)]]
    vj = ctx.vj_upper_with_rimatr_v([small.dm], 1, 1.0)[0]
    vk = ctx.vk_upper_with_ri_v([eig], [5], occ, 1, -0.5)[0]
    assert _maxdiff(vj, O.vj_upper_with_rimatr_v(small.rimatr, [small.dm], 1, 1.0)[0]) <= TOL
    ri3 = O.ri3fn_from_rimatr(small.rimatr, 37)
    assert _maxdiff(vk, O.vk_upper_with_ri_v(ri3, [eig], [5], occ, 1, -0.5)[0]) <= TOL


def test_vk_occupied_form_over_many_aux_chunks(monkeypatch):
    """A 2 MiB scratch budget splits the aux rows into chunks of 31 (n=200,
    o=33): each chunk's half-transformed orbitals sit back to back without
    padding, the rank update's k tiles straddle aux rows, and its splits end
    on partial k4 steps.  RHF and UHF K against the oracle."""
    from rest_b200 import RIJK

    monkeypatch.setenv("RIJK_SCRATCH_BYTES", str(2 << 20))
    n, naux, nocc = 200, 800, 33
    case = host_case(n, naux, nocc, seed=77)
    c2, _ = _second_spin(case, 78)
    ri3 = O.ri3fn_from_rimatr(case.rimatr, n)
    e1 = np.zeros((n, nocc + 1), order="F")
    e1[:, :nocc] = case.c_occ
    e2 = np.zeros((n, nocc + 1), order="F")
    e2[:, : c2.shape[1]] = c2
    occ1 = np.r_[np.full(nocc, 2.0), 0.0]
    occ2 = np.r_[np.full(c2.shape[1], 1.0), np.zeros(nocc + 1 - c2.shape[1])]
    c = RIJK(0)
    try:
        c.set_rimatr(case.rimatr, n)
        for spin, scale in ((1, -0.5), (2, -1.0)):
            eig, homo, occ = [e1, e2][:spin], [nocc - 1, c2.shape[1] - 1][:spin], [occ1, occ2][:spin]
            got = c.vk_upper_with_ri_v(eig, homo, occ, spin, scale)
            ref = O.vk_upper_with_ri_v(ri3, eig, homo, occ, spin, scale)
            for s in range(spin):
                assert _maxdiff(got[s], ref[s]) <= TOL
    finally:
        c.close()


def _k_occ_from_rimatr(rimatr, n, c, occ):
    """Oracle occupied-form K (REST vk_upper_with_ri_v_sync, scf_io/mod.rs:2758-2834)
    straight from rimatr, one aux row at a time: X = B_P C, K += X occ X^T."""
    ii, jj = O.upper_pairs(n)
    k = np.zeros((n, n))
    bp = np.zeros((n, n))
    for p in range(rimatr.shape[1]):
        bp[ii, jj] = rimatr[:, p]
        bp[jj, ii] = rimatr[:, p]
        x = bp @ c
        k += (x * occ) @ x.T
    return k[ii, jj]


@pytest.mark.parametrize("scratch", [None, 50 << 20])
def test_benched_shape_n1200_aux_slab_against_oracle(monkeypatch, scratch):
    """The benchmark's shape (n=1200, nocc=200) element-wise against the oracle.

    The first 96 aux rows of the n=1200, N=4800 sweep tensor (the same NumPy
    draw as the full tensor's rows) are loaded as rimatr.  At n=1200 the last
    row block of every B_P holds 48 of 64 rows and at nocc=200 the last column
    block of the half-transform holds 8 of 64 orbitals, so the straddling
    warp tiles of the DMMA mainloop run on every aux row.  With a 50 MiB
    scratch budget the 96 rows split into chunks of 25 (4 chunks, the last one
    ragged).  RHF J (a2) and K (a3), and UHF K with a second spin of 150
    orbitals, must equal the oracle within 1e-10 per element."""
    from rest_b200 import RIJK

    if scratch is not None:
        monkeypatch.setenv("RIJK_SCRATCH_BYTES", str(scratch))
    n, naux, nocc = 1200, 4800, 200
    case = host_case(n, naux, nocc, seed=2024, rows=(0, 96))
    assert case.rimatr.shape == (n * (n + 1) // 2, 96)
    rng = np.random.default_rng(12)
    c2 = np.asfortranarray(np.linalg.qr(rng.standard_normal((n, 150)))[0])
    c = RIJK(0)
    try:
        c.set_rimatr(case.rimatr, n)
        j = c.vj_upper_with_rimatr_v([case.dm], 1, 1.0)[0]
        assert _maxdiff(j, O.vj_upper_with_rimatr_v(case.rimatr, [case.dm], 1, 1.0)[0]) <= TOL
        occ1 = np.full(nocc, 2.0)
        k = c.vk_upper_with_ri_v([case.c_occ], [nocc - 1], [occ1], 1, -0.5)[0]
        k_ref = _k_occ_from_rimatr(case.rimatr, n, case.c_occ, occ1)
        assert _maxdiff(k, -0.5 * k_ref) <= TOL
        e2 = np.zeros((n, nocc), order="F")
        e2[:, :150] = c2
        occ2 = np.r_[np.ones(150), np.zeros(nocc - 150)]
        ku = c.vk_upper_with_ri_v([case.c_occ, e2], [nocc - 1, 149], [0.5 * occ1, occ2], 2, -1.0)
        assert _maxdiff(ku[0], -0.5 * k_ref) <= TOL
        assert _maxdiff(ku[1], -_k_occ_from_rimatr(case.rimatr, n, c2, np.ones(150))) <= TOL
    finally:
        c.close()


@pytest.mark.parametrize("n,naux,occs", [(150, 300, (72,)), (130, 260, (80,)), (100, 200, (65,)), (137, 200, (64, 10)),
                                         (97, 150, (60, 7))])
def test_vk_remainder_columns_of_the_last_full_block(ctx, n, naux, occs):
    """Valid orbital columns ending 1..16 past a multiple of 64 are computed by
    the last full column block's CTAs (one or two extra fragments staged in the
    slot padding); RHF and UHF K against the oracle."""
    case = host_case(n, naux, 2, seed=500 + n)
    ctx.set_rimatr(case.rimatr, n)
    ri3 = O.ri3fn_from_rimatr(case.rimatr, n)
    rng = np.random.default_rng(n)
    spin = len(occs)
    num_state = max(occs) + 1
    eig, homo, occ = [], [], []
    for s, o in enumerate(occs):
        c = np.asfortranarray(np.linalg.qr(rng.standard_normal((n, o)))[0])
        e = np.zeros((n, num_state), order="F")
        e[:, :o] = c
        eig.append(e)
        homo.append(o - 1)
        occ.append(np.r_[np.linspace(0.5, 2.0 / spin, o), np.zeros(num_state - o)])
    got = ctx.vk_upper_with_ri_v(eig, homo, occ, spin, -0.5 if spin == 1 else -1.0)
    ref = O.vk_upper_with_ri_v(ri3, eig, homo, occ, spin, -0.5 if spin == 1 else -1.0)
    for s in range(spin):
        assert _maxdiff(got[s], ref[s]) <= TOL
