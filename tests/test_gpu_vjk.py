"""J and K from one build (rijk_vjk_upper_occ_dev) against the FP64 oracle.

REST's SCF asks for J of the density C diag(occ) C^T and the occupied-orbital K
together (generate_hf_hamiltonian_ri_v, scf_io/mod.rs:1339-1381).  The fused
entry takes J's aux-row scalars B_P : D_s from the K half-transform's output
tiles, so its J is summed in another order than the two-pass J: the tolerance
is the FP64 contract's 1e-10 per element against the oracle, and K must equal
rijk_vk_upper_occ_dev's bit for bit (the same kernels on the same operands).
"""
import numpy as np
import pytest

from oracle import rijk_oracle as O
from rest_b200.synth import host_case

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _maxdiff(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))))


def _orbitals(n, occs, seed):
    """Per spin: eigenvectors (n x num_state, the first o columns orthonormal),
    homo and occupations (decreasing, fractional for the last states)."""
    rng = np.random.default_rng(seed)
    spin = len(occs)
    num_state = max(occs) + 2
    eig, homo, occ = [], [], []
    for o in occs:
        c = np.linalg.qr(rng.standard_normal((n, o)))[0]
        e = np.zeros((n, num_state), order="F")
        e[:, :o] = c
        e[:, o:] = rng.standard_normal((n, num_state - o))  # states above homo: ignored
        eig.append(e)
        homo.append(o - 1)
        occ.append(np.r_[np.linspace(2.0 / spin, 0.25, o), np.zeros(num_state - o)])
    return eig, homo, occ, num_state


def _fused(ctx, eig, homo, occ, num_state, spin, jscale, kscale, split=False):
    import torch

    n = eig[0].shape[0]
    npair = n * (n + 1) // 2
    d_e = torch.from_numpy(np.concatenate([np.asarray(e, order="F").ravel(order="F") for e in eig])).cuda()
    d_o = torch.from_numpy(np.concatenate(occ)).cuda()
    vj = torch.full((spin * npair,), np.nan, dtype=torch.float64, device="cuda")
    vk = torch.full((spin * npair,), np.nan, dtype=torch.float64, device="cuda")
    ctx.vjk_upper_occ_dev(d_e.data_ptr(), num_state, homo, d_o.data_ptr(), spin, jscale, kscale, vj.data_ptr(),
                          vk.data_ptr())
    ctx.synchronize()
    # the separate entries on the same device operands
    vj2 = torch.empty_like(vj)
    vk2 = torch.empty_like(vk)
    dms = []
    for s in range(spin):
        c = eig[s][:, : homo[s] + 1]
        dms.append(np.asfortranarray((c * occ[s][: homo[s] + 1]) @ c.T))
    d_dm = torch.from_numpy(np.concatenate([d.ravel(order="F") for d in dms])).cuda()
    ctx.vj_upper_dev(d_dm.data_ptr(), spin, jscale, 0, vj2.data_ptr())
    ctx.vk_upper_occ_dev(d_e.data_ptr(), num_state, homo, d_o.data_ptr(), spin, kscale, vk2.data_ptr())
    ctx.synchronize()
    split_j = lambda t: [t[s * npair:(s + 1) * npair].cpu().numpy() for s in range(spin)]  # noqa: E731
    return split_j(vj), split_j(vk), split_j(vj2), split_j(vk2), dms


@pytest.mark.parametrize("n,naux,occs", [(24, 113, (5,)), (37, 150, (6, 4)), (100, 400, (16,)), (150, 300, (72,)),
                                         (137, 200, (64, 10)), (97, 150, (60, 7)), (200, 800, (33, 32))])
def test_vjk_against_oracle_and_separate_entries(ctx, n, naux, occs):
    case = host_case(n, naux, 2, seed=700 + n)
    ctx.set_rimatr(case.rimatr, n)
    ri3 = O.ri3fn_from_rimatr(case.rimatr, n)
    eig, homo, occ, num_state = _orbitals(n, occs, n + 7)
    spin = len(occs)
    kscale = -0.5 if spin == 1 else -1.0
    vj, vk, vj2, vk2, dms = _fused(ctx, eig, homo, occ, num_state, spin, 1.0, kscale)
    jref = O.vj_upper_with_ri_v(ri3, dms, spin, 1.0)
    kref = O.vk_upper_with_ri_v(ri3, eig, homo, occ, spin, kscale)
    for s in range(spin):
        assert _maxdiff(vj[s], jref[s]) <= TOL
        assert _maxdiff(vk[s], kref[s]) <= TOL
        assert np.array_equal(vk[s], vk2[s])
        assert _maxdiff(vj[s], vj2[s]) <= 1e-12 * max(1.0, float(np.max(np.abs(vj2[s]))))


@pytest.mark.parametrize("ht", [0, 1, 2, 3, 4, 5])
def test_every_half_transform_shape_gives_the_same_j(ctx, ht):
    """The J scalars come from the consumer warps of every CTA shape, including
    the bulk-copy shape with its producer warp."""
    n, naux = 150, 300
    case = host_case(n, naux, 2, seed=41)
    ctx.set_rimatr(case.rimatr, n)
    ri3 = O.ri3fn_from_rimatr(case.rimatr, n)
    eig, homo, occ, num_state = _orbitals(n, (40, 23), 42)
    try:
        ctx.set_tiles(ht, 1)
        vj, vk, _, vk2, dms = _fused(ctx, eig, homo, occ, num_state, 2, 2.0, -1.0)
    finally:
        ctx.set_tiles(1, 1)
    jref = O.vj_upper_with_ri_v(ri3, dms, 2, 2.0)
    for s in range(2):
        assert _maxdiff(vj[s], jref[s]) <= TOL
        assert np.array_equal(vk[s], vk2[s])


def test_vjk_over_many_aux_chunks(monkeypatch):
    """A 2 MiB scratch budget cuts the aux rows into chunks: each chunk's J
    scalars land at their own rows of w before J's second pass."""
    from rest_b200 import RIJK

    monkeypatch.setenv("RIJK_SCRATCH_BYTES", str(2 << 20))
    n, naux = 200, 800
    case = host_case(n, naux, 2, seed=81)
    ri3 = O.ri3fn_from_rimatr(case.rimatr, n)
    eig, homo, occ, num_state = _orbitals(n, (33, 30), 82)
    c = RIJK(0)
    try:
        c.set_rimatr(case.rimatr, n)
        for spin in (1, 2):
            vj, vk, _, vk2, dms = _fused(c, eig[:spin], homo[:spin], occ[:spin], num_state, spin, 1.0, -1.0)
            jref = O.vj_upper_with_ri_v(ri3, dms, spin, 1.0)
            for s in range(spin):
                assert _maxdiff(vj[s], jref[s]) <= TOL
                assert np.array_equal(vk[s], vk2[s])
    finally:
        c.close()


def test_vjk_rejects_bad_arguments(ctx):
    import torch

    from rest_b200 import RijkError

    n = 24
    case = host_case(n, 113, 5, seed=3)
    ctx.set_rimatr(case.rimatr, n)
    e = torch.zeros(n * 6, dtype=torch.float64, device="cuda")
    o = torch.ones(6, dtype=torch.float64, device="cuda")
    v = torch.zeros(n * (n + 1) // 2, dtype=torch.float64, device="cuda")
    with pytest.raises(RijkError):  # J and K into the same buffer
        ctx.vjk_upper_occ_dev(e.data_ptr(), 6, [4], o.data_ptr(), 1, 1.0, -0.5, v.data_ptr(), v.data_ptr())
    with pytest.raises(RijkError):  # homo beyond num_state
        w = torch.zeros_like(v)
        ctx.vjk_upper_occ_dev(e.data_ptr(), 6, [6], o.data_ptr(), 1, 1.0, -0.5, v.data_ptr(), w.data_ptr())


@pytest.mark.parametrize("occs", [(16,), (16, 11)])
def test_vjk_host_form_against_oracle(ctx, occs):
    """rijk_vjk_upper_with_ri_v: host buffers in and out (the call REST's SCF
    would bind for generate_hf_hamiltonian_ri_v)."""
    n, naux = 100, 400
    case = host_case(n, naux, 2, seed=91)
    ctx.set_rimatr(case.rimatr, n)
    ri3 = O.ri3fn_from_rimatr(case.rimatr, n)
    eig, homo, occ, _ = _orbitals(n, occs, 92)
    spin = len(occs)
    vj, vk = ctx.vjk_upper_with_ri_v(eig, homo, occ, spin, 1.0, -0.5 if spin == 1 else -1.0)
    dms = []
    for s in range(spin):
        c = eig[s][:, : homo[s] + 1]
        dms.append(np.asfortranarray((c * occ[s][: homo[s] + 1]) @ c.T))
    jref = O.vj_upper_with_ri_v(ri3, dms, spin, 1.0)
    kref = O.vk_upper_with_ri_v(ri3, eig, homo, occ, spin, -0.5 if spin == 1 else -1.0)
    for s in range(spin):
        assert _maxdiff(vj[s], jref[s]) <= TOL
        assert _maxdiff(vk[s], kref[s]) <= TOL
