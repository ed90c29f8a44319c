"""Learned-guess pieces that need no GPU: the frame / rotation machinery and the
MLP oracle itself (finite differences)."""
import numpy as np

from oracle import mlp_oracle as mo
from rest_b200.basis import ANG, Molecule, int1e
from rest_b200.geometry import water_cluster
from rest_b200.guess import assemble_density, local_blocks, pair_features, shell_rotation


def test_shell_rotations_are_orthogonal():
    rng = np.random.default_rng(0)
    q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
    q[:, 0] *= np.sign(np.linalg.det(q))
    for l in range(3):
        g = shell_rotation(l, q)
        assert np.abs(g @ g.T - np.eye(2 * l + 1)).max() < 1e-12


def test_features_and_local_blocks_are_rotation_invariant():
    """The overlap matrix transforms like a density: its blocks in the water
    frames must not change under a rigid motion of the cluster."""
    mol = water_cluster(3, seed=1)
    rng = np.random.default_rng(3)
    q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
    q[:, 0] *= np.sign(np.linalg.det(q))
    xyz = np.asarray(mol.coords) * ANG
    moved = Molecule.from_angstrom(mol.symbols, xyz @ q.T + np.array([1.0, -2.0, 0.5]))
    out = []
    for m in (mol, moved):
        sh = m.shells("def2-SVP")
        ps = pair_features(m)
        t, _ = local_blocks(m, sh, int1e(m, sh, "ovlp"), ps)
        out.append((ps.feats, t))
    assert np.abs(out[0][0] - out[1][0]).max() < 1e-12
    assert np.abs(out[0][1] - out[1][1]).max() < 1e-12


def test_blocks_round_trip_within_cutoff():
    mol = water_cluster(4, seed=2)
    sh = mol.shells("def2-SVP")
    rng = np.random.default_rng(1)
    a = rng.standard_normal((sh.nfun, sh.nfun))
    d = a + a.T
    ps = pair_features(mol)
    t, _ = local_blocks(mol, sh, d, ps)
    back = assemble_density(mol, sh, ps, t)
    xyz = np.asarray(mol.coords) * ANG
    atom_of = np.repeat(np.arange(len(mol.symbols)), [14 if s == "O" else 5 for s in mol.symbols])
    dist = np.linalg.norm(xyz[atom_of][:, None] - xyz[atom_of][None], axis=-1)
    ref = np.where(dist <= 6.0, d, 0.0)
    assert np.abs(back - ref).max() < 1e-12


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 1e-30], dtype=np.float32)
    v = mo.round_bf16(x)
    assert v[0] == 1.0 and v[1] == 1.0  # tie to even
    assert v[2] == 1.0 + 2 ** -6  # tie to even (upwards)
    assert v[3] == -2.5


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(5)
    dims = [7, 9, 6, 5]
    ws = [rng.standard_normal((n, k)) * 0.5 for k, n in zip(dims[:-1], dims[1:])]
    bs = [rng.standard_normal(n) * 0.1 for n in dims[1:]]
    x = rng.standard_normal((11, dims[0]))
    t = rng.standard_normal((11, dims[-1]))
    mask = (rng.random((11, dims[-1])) > 0.3).astype(float)
    loss, grads = mo.network_loss_and_grads(x, ws, bs, t, mask, 13.0)
    h = 1e-6
    for li in range(len(ws)):
        for (i, j) in [(0, 0), (ws[li].shape[0] - 1, ws[li].shape[1] - 1), (1, 2)]:
            wp = [w.copy() for w in ws]
            wp[li][i, j] += h
            wm = [w.copy() for w in ws]
            wm[li][i, j] -= h
            fd = (mo.network_loss_and_grads(x, wp, bs, t, mask, 13.0)[0]
                  - mo.network_loss_and_grads(x, wm, bs, t, mask, 13.0)[0]) / (2 * h)
            assert abs(fd - grads[li][0][i, j]) < 1e-7 * max(1.0, abs(fd))


def test_pair_layout_and_row_arithmetic_match_host_assembly_inputs():
    """The host half of the device geometry (pair_layout) and, restated in
    NumPy, the row arithmetic of the pair kernel (rows at the exclusive scan of
    the neighbour counts; the row of (B, A) from B's neighbours before A) give
    the host assembly inputs of every molecule of a set of uneven sizes."""
    from rest_b200.guess import CUTOFF, assembly_inputs, geometry_table, pair_layout

    mols = [water_cluster(k, seed=40 + k) for k in (1, 4, 2, 9)]
    lo = pair_layout(mols, "def2-SVP")
    assert geometry_table().size == 516
    assert list(lo.elem_shells[0, :7]) == [6, 0, 0, 0, 1, 1, 2] and list(lo.elem_shells[1, :4]) == [3, 0, 0, 1]
    for i, m in enumerate(mols):
        a0, a1 = lo.atom_off[i], lo.atom_off[i + 1]
        sh = m.shells("def2-SVP")
        ps = pair_features(m)
        up, first, typ, nfun, water, _ = assembly_inputs(m, sh, ps)
        for got, want in ((lo.first, first), (lo.typ, typ), (lo.nfun, nfun), (lo.water, water)):
            assert np.array_equal(got[a0:a1], want)
        assert lo.nbas[i] == sh.nfun
        assert np.all(lo.info[a0:a1, 0] == a0) and np.all(lo.info[a0:a1, 1] == a1 - a0)
        x = lo.xyz[a0:a1]
        near = np.linalg.norm(x[:, None] - x[None], axis=-1) <= CUTOFF
        off = np.concatenate([[0], np.cumsum(near.sum(axis=1))])
        rows = []
        for a in range(a1 - a0):
            nb = np.nonzero(near[a])[0]
            for r, b in enumerate(nb):
                if b >= a:
                    rows.append((a, b, off[a] + r, off[b] + int(near[b, :a].sum())))
        assert np.array_equal(np.array(rows, dtype=np.int32), up)


def test_pair_layout_refuses_what_the_geometry_kernels_cannot_take():
    """The host checks in front of rijk_guess_geometry: atoms not ordered O, H, H
    per water, an empty molecule or set, and element blocks beyond 14 functions
    or l > 2 are refused before anything reaches the device."""
    import pytest

    from rest_b200.guess import pair_layout

    bad_order = Molecule.from_angstrom(["H", "O", "H"], [[0, 0, 0], [0, 0, 1], [0, 1, 0]])
    empty = Molecule.from_angstrom([], np.zeros((0, 3)))
    water = water_cluster(2, seed=1)
    for mols in ([bad_order], [water, empty], []):
        with pytest.raises(ValueError):
            pair_layout(mols, "def2-SVP")
    with pytest.raises(ValueError, match="14 functions"):
        pair_layout([water], "aug-cc-pV5Z")
