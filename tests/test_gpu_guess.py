"""Learned initial guess on the GPU: the MLP kernels (rijk_mlp_*) against the
CPU oracle (oracle/mlp_oracle.py), training on converged densities, and the
trained network's effect on the SCF.

Tolerances: single layers agree with the oracle to 1e-5 of the largest element
(FP32 against float64 sums of identical BF16 operands; 2e-3 where the SiLU
derivative is rounded to BF16 on both sides and may round the other way); the
whole-network gradient, whose hidden activations are BF16 on the device only,
to 3 % in norm.
"""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import mlp_oracle as mo
from rest_b200._abi import lib
from rest_b200.geometry import water_cluster
from rest_b200.guess import DEFAULT_WEIGHTS, LAYERS, LearnedGuess, PairMLP, train
from rest_b200.scf_batch import run_molecule_set

pytestmark = pytest.mark.gpu


def _dev(a, dtype):
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _bits(a):
    return torch.tensor(mo.bf16_bits(a).view(np.int16), device="cuda")


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _close(got, ref, tol):
    return np.abs(np.asarray(got, np.float64) - ref).max() <= tol * max(np.abs(ref).max(), 1e-30)


@pytest.mark.parametrize("m,k,n,act", [(1, 3, 5, 0), (37, 53, 256, 1), (300, 256, 196, 0), (129, 70, 64, 1)])
def test_linear_forward_matches_oracle(m, k, n, act):
    rng = np.random.default_rng(m + k + n)
    x, w, b = rng.standard_normal((m, k)), rng.standard_normal((n, k)) * 0.2, rng.standard_normal(n)
    xb, wb = mo.bf16_bits(x), mo.bf16_bits(w)
    z_ref, y_ref = mo.linear_fwd(xb, wb, b.astype(np.float32), act)
    z = torch.empty(m, n, dtype=torch.float32, device="cuda")
    y = torch.empty(m, n, dtype=torch.float32, device="cuda")
    yb = torch.empty(m, n, dtype=torch.int16, device="cuda")
    xd, wd, bd = _bits(x), _bits(w), _dev(b, torch.float32)  # operands stay alive until the launch
    st = lib().rijk_mlp_linear_fwd(_p(xd), _p(wd), _p(bd), m, k, n, act, _p(z), _p(yb), _p(y), None)
    assert st == 0
    torch.cuda.synchronize()
    assert _close(z.cpu().numpy(), z_ref, 1e-5)
    assert _close(y.cpu().numpy(), y_ref, 1e-5)
    assert np.array_equal(yb.cpu().numpy().view(np.uint16), mo.bf16_bits(y.cpu().numpy()))


@pytest.mark.parametrize("m,k,n,act,tol", [(64, 53, 256, 0, 1e-5), (4096, 256, 196, 0, 1e-5), (333, 256, 256, 1, 2e-3)])
def test_linear_backward_matches_oracle(m, k, n, act, tol):
    rng = np.random.default_rng(m + n)
    x, w = rng.standard_normal((m, k)), rng.standard_normal((n, k)) * 0.1
    z, dy = rng.standard_normal((m, n)).astype(np.float32), rng.standard_normal((m, n)).astype(np.float32)
    dw_ref, db_ref, dx_ref, _ = mo.linear_bwd(mo.bf16_bits(x), mo.bf16_bits(w), z, dy, act)
    dz = torch.empty(m, n, dtype=torch.int16, device="cuda")
    dw = torch.empty(n, k, dtype=torch.float32, device="cuda")
    db = torch.empty(n, dtype=torch.float32, device="cuda")
    dx = torch.empty(m, k, dtype=torch.float32, device="cuda")
    xd, wd, zd, dyd = _bits(x), _bits(w), _dev(z, torch.float32), _dev(dy, torch.float32)
    st = lib().rijk_mlp_linear_bwd(_p(xd), _p(wd), _p(zd), _p(dyd), m, k, n, act, _p(dz), _p(dw), _p(db), _p(dx),
                                   None)
    assert st == 0
    torch.cuda.synchronize()
    assert _close(dw.cpu().numpy(), dw_ref, tol)
    assert _close(db.cpu().numpy(), db_ref, tol)
    assert _close(dx.cpu().numpy(), dx_ref, tol)


def test_masked_mse_and_adam_match_oracle():
    rng = np.random.default_rng(9)
    y, t = rng.standard_normal(5000).astype(np.float32), rng.standard_normal(5000).astype(np.float32)
    mask = (rng.random(5000) > 0.4).astype(np.float32)
    loss_ref, dy_ref = mo.masked_mse(y, t, mask, float(mask.sum()))
    dy = torch.empty(5000, dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    yd, td, md = _dev(y, torch.float32), _dev(t, torch.float32), _dev(mask, torch.float32)
    assert lib().rijk_mlp_masked_mse(_p(yd), _p(td), _p(md), 5000, float(mask.sum()), _p(dy), _p(loss), None) == 0
    torch.cuda.synchronize()
    assert abs(float(loss) - loss_ref) <= 1e-5 * loss_ref
    assert _close(dy.cpu().numpy(), dy_ref, 1e-6)
    w0 = rng.standard_normal(777)
    w, m, v = w0.copy(), np.zeros(777), np.zeros(777)
    dw_, dm_, dv_ = _dev(w0, torch.float32), torch.zeros(777, device="cuda"), torch.zeros(777, device="cuda")
    wbf = torch.empty(777, dtype=torch.int16, device="cuda")
    for step in range(1, 4):
        g = rng.standard_normal(777)
        w, m, v = mo.adam(w, g, m, v, 1e-2, 0.9, 0.999, 1e-8, step)
        gd = _dev(g, torch.float32)
        assert lib().rijk_mlp_adam(_p(dw_), _p(wbf), _p(gd), _p(dm_), _p(dv_), 777, 1e-2, 0.9, 0.999, 1e-8, step,
                                   None) == 0
        torch.cuda.synchronize()
    torch.cuda.synchronize()
    assert _close(dw_.cpu().numpy(), w, 1e-5)
    assert np.array_equal(wbf.cpu().numpy().view(np.uint16), mo.bf16_bits(dw_.cpu().numpy()))


def test_network_gradient_matches_oracle():
    net = PairMLP(layers=[53, 64, 64, 32], seed=3)
    rng = np.random.default_rng(4)
    x = rng.standard_normal((200, 53))
    t = rng.standard_normal((200, 32)) * 0.3
    mask = (rng.random((200, 32)) > 0.2).astype(np.float64)
    xb, td, md = _bits(x), _dev(t, torch.float32), _dev(mask, torch.float32)
    loss, grads = net.gradients(xb, td, md, float(mask.sum()))
    torch.cuda.synchronize()
    ws = [mo.round_bf16(w.cpu().numpy()) for w in net.W]
    bs = [b.cpu().numpy().astype(np.float64) for b in net.b]
    loss_ref, grads_ref = mo.network_loss_and_grads(mo.round_bf16(x), ws, bs, t, mask, float(mask.sum()))
    assert abs(float(loss) - loss_ref) <= 1e-2 * loss_ref
    for (dw, db), (dw_r, db_r) in zip(grads, grads_ref):
        for got, ref in ((dw.cpu().numpy(), dw_r), (db.cpu().numpy(), db_r)):
            assert np.linalg.norm(got - ref) <= 3e-2 * np.linalg.norm(ref)


def test_training_on_converged_densities_lowers_the_loss():
    mols = [water_cluster(k, seed=300 + k) for k in (1, 2, 3, 2, 1)]
    res = run_molecule_set(mols, "def2-SVP", "def2-SVP-JKFIT", group_size=5, return_densities=True,
                           acc_etot=1e-8, acc_rho=1e-6, acc_eev=1e-6)
    assert all(res.converged)
    net, norm, hist = train(list(zip(mols, res.densities)), epochs=40, batch=64, lr=2e-3, seed=0)
    assert hist[-1] < 0.2 * hist[0]
    assert [w.shape[1] for w in net.W] == LAYERS[:-1]


@pytest.mark.skipif(not Path(DEFAULT_WEIGHTS).exists(), reason="no trained weights committed")
def test_committed_guess_cuts_scf_iterations_on_held_out_clusters():
    """Held-out clusters larger than any training cluster (k = 13..16): the
    learned density must start the SCF closer than REST's hcore guess and reach
    the same FP64 energy."""
    from rest_b200.basis import int1e

    guess = LearnedGuess.load()
    mols = [water_cluster(k, seed=9000 + k) for k in (13, 14, 15, 16)]
    crit = dict(acc_etot=1e-8, acc_rho=1e-6, acc_eev=1e-6, max_cycle=100)
    ref = run_molecule_set(mols, "def2-SVP", "def2-SVP-JKFIT", group_size=4, **crit)
    dens = [guess.density(m, ovlp=int1e(m, m.shells("def2-SVP"), "ovlp")) for m in mols]
    assert all(d is not None for d in dens)
    lrn = run_molecule_set(mols, "def2-SVP", "def2-SVP-JKFIT", group_size=4, initial_densities=dens, **crit)
    assert all(ref.converged) and all(lrn.converged)
    assert np.mean(lrn.iterations) < np.mean(ref.iterations)
    assert np.max(np.abs(np.array(lrn.energies) - np.array(ref.energies))) < 1e-6


def test_learned_density_handed_to_rest_as_init_guess(tmp_path):
    """The learned density written as REST's init_guess file (REST's AO order)
    reads back as the same density and holds the cluster's electrons."""
    from rest_b200.basis import int1e
    from rest_b200.chkfile import H5Reader, read_init_guess, rest_ao_order

    guess = LearnedGuess.load()
    mol = water_cluster(5, seed=77)
    sh = mol.shells(guess.basis)
    s = int1e(mol, sh, "ovlp")
    path = tmp_path / "init_guess.chk"
    assert guess.write_rest_init_guess(mol, path, ovlp=s)
    d = guess.density(mol, ovlp=s)
    back = read_init_guess(path, sh.nfun, 1, shells=sh)[0]
    assert np.array_equal(back, d)
    raw = H5Reader.open(path).dataset("init_guess")
    perm = rest_ao_order(sh)
    assert np.array_equal(raw.T, d[np.ix_(perm, perm)])  # column-major, REST's AO order
    assert abs(float(np.sum(back * s)) - mol.nelec) < 1e-8


@pytest.mark.parametrize("k", [1, 4, 13])
def test_device_assembly_matches_host_assembly(k):
    """rijk_guess_assemble (per unordered pair, both water frames, no atomics)
    against the NumPy assembly of the same network output."""
    from rest_b200.guess import assemble_density, pair_features

    guess = LearnedGuess.load()
    mol = water_cluster(k, seed=90 + k)
    sh = mol.shells(guess.basis)
    ps = pair_features(mol)
    y = guess._forward(ps)
    ref = assemble_density(mol, sh, ps, guess.norm.blocks(y.cpu().numpy().astype(np.float64), ps.kind))
    got = guess.assemble_device(mol, sh, ps, y).cpu().numpy()
    assert np.max(np.abs(got - ref)) <= 1e-6 * np.max(np.abs(ref))
    assert np.array_equal(got, got.T)


def test_device_pair_rows_match_host():
    """rijk_guess_geometry + rijk_guess_pairs over a molecule set of uneven
    sizes against the host restatement (pair_features, Rotator,
    assembly_inputs): the same pairs in the same order, the same unordered-pair
    rows, layout and rotations; features equal to FP32 rounding of the
    standardised values."""
    from rest_b200.guess import Rotator, assembly_inputs, device_pairs, pair_features, water_frames

    guess = LearnedGuess.load()
    mols = [water_cluster(k, seed=300 + k) for k in (1, 2, 7, 16, 3, 24)]
    g = device_pairs(mols, guess.basis, guess.norm, torch.device("cuda"))
    feats, up = g.feats.cpu().numpy(), g.up.cpu().numpy()
    rot = g.rot.cpu().numpy()
    lay = [t.cpu().numpy() for t in (g.first, g.typ, g.nfun, g.water)]
    for i, m in enumerate(mols):
        sh = m.shells(guess.basis)
        fr = water_frames(m)
        ps = pair_features(m, fr)
        r = Rotator(m, sh, fr)
        h_up, h_first, h_typ, h_nfun, h_water, h_rot = assembly_inputs(m, sh, ps, r)
        p0, p1 = g.pair_off[i], g.pair_off[i + 1]
        a0, a1 = g.atom_off[i], g.atom_off[i + 1]
        assert p1 - p0 == len(ps.pairs) and g.nbas[i] == sh.nfun
        ref = guess.norm.feats(ps.feats)
        assert np.max(np.abs(feats[p0:p1] - ref)) <= 2e-6 * max(1.0, np.abs(ref).max())
        assert np.array_equal(up[g.up_off[i]:g.up_off[i + 1]], h_up)
        for got, want in zip(lay, (h_first, h_typ, h_nfun, h_water)):
            assert np.array_equal(got[a0:a1], want)
        assert np.max(np.abs(rot[a0 // 3:a1 // 3] - h_rot)) <= 1e-12


def test_batched_densities_match_single_molecule_path():
    """densities() over a set (device pair rows, one network pass) gives each
    molecule the density of the host-feature path for that molecule alone, and
    the electron-count check scales it to the molecule's electrons."""
    from rest_b200.basis import int1e
    from rest_b200.guess import pair_features

    guess = LearnedGuess.load()
    mols = [water_cluster(k, seed=500 + k) for k in (2, 9, 16, 5)]
    ovl = [int1e(m, m.shells(guess.basis), "ovlp") for m in mols]
    got = guess.densities(mols, ovl)
    for m, s, d in zip(mols, ovl, got):
        sh = m.shells(guess.basis)
        ps = pair_features(m)
        ref = guess.assemble_device(m, sh, ps, guess._forward(ps)).cpu().numpy()
        ref *= m.nelec / float(np.sum(ref * s))
        assert d is not None
        assert np.max(np.abs(d.cpu().numpy() - ref)) <= 1e-10 * np.max(np.abs(ref))
        assert abs(float(np.sum(d.cpu().numpy() * s)) - m.nelec) < 1e-9
