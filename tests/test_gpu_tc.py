"""Split-precision (3 x BF16 on tcgen05) exchange against the FP64 path.

* exact: integer-valued tensors and orbitals that BF16 holds exactly give the
  FP64 result bit for bit (checks every layout and descriptor of the kernels);
* accurate: random data agree with the FP64 build to 1e-4 of max |K|
  (the split keeps ~17 of the 53 mantissa bits);
* signed low-rank: K of a density difference V S V^T equals the FP64
  density-form K of that difference to the same relative accuracy.
"""
import numpy as np
import pytest

from oracle import rijk_oracle as O
from rest_b200.synth import host_case

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch

    return torch.tensor(np.asarray(a), dtype=torch.float64, device="cuda")


def _split_k_occ(ctx, c, occ):
    import torch

    n, nocc = c.shape
    st = ctx.stream
    with torch.cuda.stream(torch.cuda.ExternalStream(st)):
        dc = _dev(np.asfortranarray(c).T.copy())  # column-major n x nocc
        do = _dev(occ)
        out = torch.empty(n * (n + 1) // 2, dtype=torch.float64, device="cuda")
        ctx.vk_upper_occ_split_dev(dc.data_ptr(), nocc, [nocc - 1], do.data_ptr(), 1, 1.0, out.data_ptr(), st)
        ctx.synchronize(st)
        return out.cpu().numpy()


@pytest.mark.parametrize("env", [{}, {"RIJK_TC_PAIR": "1"}, {"RIJK_TC_PAIR": "0", "RIJK_TC_KS": "32"}])
@pytest.mark.parametrize("n,naux,nocc", [(64, 24, 8), (100, 40, 16), (200, 30, 40), (300, 20, 24), (520, 6, 72),
                                         (100, 41, 16), (520, 7, 72), (200, 31, 160), (390, 9, 130)])
def test_split_exchange_is_exact_on_bf16_representable_input(ctx, monkeypatch, env, n, naux, nocc):
    """Every kernel form: the defaults (one SM per tile with K 64 per stage,
    the half-transform on SM pairs from five 128-row blocks on and the rank
    update from six), both
    kernels on SM pairs (cta_group::2), and one SM each with K 32 per stage; odd
    aux counts (a pair whose second aux row is missing), odd 128-row block
    counts (K block groups with rows beyond n) and every column padding (64,
    128, 256)."""
    monkeypatch.delenv("RIJK_TC_PAIR", raising=False)
    monkeypatch.delenv("RIJK_TC_KS", raising=False)
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    rng = np.random.default_rng(n)
    npair = n * (n + 1) // 2
    rimatr = np.asfortranarray(rng.integers(-1, 2, size=(npair, naux)).astype(np.float64))
    c = np.asfortranarray(rng.integers(-1, 2, size=(n, nocc)).astype(np.float64))
    occ = np.ones(nocc)
    ctx.set_rimatr(rimatr, n)
    got = _split_k_occ(ctx, c, occ)
    ref = ctx.vk_upper_with_ri_v([c], [nocc - 1], [occ], 1, 1.0)[0]
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("n,naux,nocc", [(150, 600, 25), (300, 1200, 50), (600, 2400, 100)])
def test_split_exchange_accuracy(ctx, n, naux, nocc):
    case = host_case(n, naux, nocc, seed=11 + n)
    ctx.set_rimatr(case.rimatr, n)
    occ = np.full(nocc, 2.0)
    got = _split_k_occ(ctx, case.c_occ, occ)
    ref = ctx.vk_upper_with_ri_v([case.c_occ], [nocc - 1], [occ], 1, 1.0)[0]
    assert np.max(np.abs(got - ref)) <= 1e-4 * np.max(np.abs(ref))


@pytest.mark.parametrize("n,naux,npos,nneg", [(120, 480, 20, 12), (260, 1000, 300, 40)])
def test_split_lowrank_signed(ctx, n, naux, npos, nneg):
    import torch

    case = host_case(n, naux, 4, seed=5 + n)
    ctx.set_rimatr(case.rimatr, n)
    rng = np.random.default_rng(n)
    v = rng.standard_normal((n, npos + nneg)) / np.sqrt(n)
    s = np.concatenate([np.ones(npos), -np.ones(nneg)])
    dd = (v * s) @ v.T
    ref = ctx.vk_upper_with_rimatr_use_dm_only([dd], 1, 1.0)[0]
    st = ctx.stream
    ld = n + (n & 1)
    vp = np.zeros((ld, npos + nneg))
    vp[:n] = v
    with torch.cuda.stream(torch.cuda.ExternalStream(st)):
        dv = _dev(np.asfortranarray(vp).T.copy())
        out = torch.empty(n * (n + 1) // 2, dtype=torch.float64, device="cuda")
        ctx.vk_upper_lowrank_split_dev(dv.data_ptr(), ld, npos + nneg, npos, 1.0, False, out.data_ptr(), st)
        ctx.synchronize(st)
        got = out.cpu().numpy()
    assert np.max(np.abs(got - ref)) <= 1e-4 * np.max(np.abs(ref))


@pytest.mark.parametrize("env", [{}, {"RIJK_TC_PAIR": "1"}])
@pytest.mark.parametrize("n,naux,npos,nneg,exact", [(120, 41, 20, 12, True), (200, 30, 150, 0, True),
                                                    (260, 1000, 300, 40, False), (390, 500, 64, 70, False)])
def test_split_lowrank_j_and_k(ctx, monkeypatch, env, n, naux, npos, nneg, exact):
    """rijk_vjk_upper_lowrank_split_dev: J of dD = V S V^T from the split
    half-transform's epilogue and K of the same difference, against the FP64
    density-form builds; bit for bit on integer-valued input (every product and
    sum exact), else within 1e-4 of max |J| and |K|; with the half-transform on
    one SM per tile and on SM pairs (odd aux counts: a pair without its second
    row)."""
    monkeypatch.delenv("RIJK_TC_PAIR", raising=False)
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    import torch

    rng = np.random.default_rng(n + naux)
    if exact:
        npair = n * (n + 1) // 2
        rimatr = np.asfortranarray(rng.integers(-1, 2, size=(npair, naux)).astype(np.float64))
        v = rng.integers(-1, 2, size=(n, npos + nneg)).astype(np.float64)
    else:
        rimatr = host_case(n, naux, 4, seed=9 + n).rimatr
        v = rng.standard_normal((n, npos + nneg)) / np.sqrt(n)
    ctx.set_rimatr(rimatr, n)
    s = np.concatenate([np.ones(npos), -np.ones(nneg)])
    dd = (v * s) @ v.T
    jref = ctx.vj_upper_with_rimatr_v([dd], 1, 1.0)[0]
    kref = ctx.vk_upper_with_rimatr_use_dm_only([dd], 1, 1.0)[0]
    st = ctx.stream
    ld = n + (n & 1)
    vp = np.zeros((ld, npos + nneg))
    vp[:n] = v
    with torch.cuda.stream(torch.cuda.ExternalStream(st)):
        dv = _dev(np.asfortranarray(vp).T.copy())
        vj = torch.full((n * (n + 1) // 2,), np.nan, dtype=torch.float64, device="cuda")
        vk = torch.empty(n * (n + 1) // 2, dtype=torch.float64, device="cuda")
        ctx.vjk_upper_lowrank_split_dev(dv.data_ptr(), ld, npos + nneg, npos, 1.0, 1.0, False, vj.data_ptr(),
                                        vk.data_ptr(), st)
        ctx.synchronize(st)
        gj, gk = vj.cpu().numpy(), vk.cpu().numpy()
    if exact:
        assert np.array_equal(gj, jref)
        assert np.array_equal(gk, kref)
    else:
        assert np.max(np.abs(gj - jref)) <= 1e-4 * np.max(np.abs(jref))
        assert np.max(np.abs(gk - kref)) <= 1e-4 * np.max(np.abs(kref))
