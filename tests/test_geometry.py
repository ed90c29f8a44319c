"""Synthetic molecule generators (CPU): alkane geometry and basis sizes of the
precision config, water-cluster constraints of the batched config."""
import numpy as np
import pytest

from rest_b200.geometry import alkane, alkane_coords, water_cluster


@pytest.mark.parametrize("nc", [1, 2, 3, 10])
def test_alkane_is_ideal_all_trans(nc):
    sym, xyz = alkane_coords(nc)
    assert sym.count("C") == nc and sym.count("H") == 2 * nc + 2
    tetra = np.degrees(np.arccos(-1.0 / 3.0))
    for i, s in enumerate(sym):
        if s != "C":
            continue
        d = np.linalg.norm(xyz - xyz[i], axis=1)
        nb = [j for j in range(len(sym)) if j != i and d[j] < 1.6]
        assert len(nb) == 4
        for j in nb:
            assert abs(d[j] - (1.54 if sym[j] == "C" else 1.09)) < 1e-12
        v = [(xyz[j] - xyz[i]) / d[j] for j in nb]
        for a in range(4):
            for b in range(a + 1, 4):
                assert abs(np.degrees(np.arccos(np.clip(v[a] @ v[b], -1, 1))) - tetra) < 1e-6


@pytest.mark.parametrize("nc,n,naux,nocc", [(10, 250, 1146, 41), (20, 490, 2256, 81), (40, 970, 4476, 161)])
def test_alkane_basis_sizes(nc, n, naux, nocc):
    mol = alkane(nc)
    assert mol.shells("def2-SVP").nfun == n
    assert mol.shells("def2-SVP-JKFIT").nfun == naux
    assert mol.nelec // 2 == nocc


def test_water_cluster_constraints():
    mol = water_cluster(12, seed=3)
    assert mol.shells("def2-SVP").nfun == 24 * 12
    xyz = np.asarray(mol.coords) * 0.5291772083  # bohr -> A
    oxy = xyz[0::3]
    d = np.linalg.norm(oxy[:, None] - oxy[None], axis=-1) + np.eye(len(oxy)) * 10
    assert d.min() >= 2.7 - 1e-9
    for w in range(12):
        o, h1, h2 = xyz[3 * w:3 * w + 3]
        assert abs(np.linalg.norm(h1 - o) - 0.9572) < 1e-9
        cosang = (h1 - o) @ (h2 - o) / np.linalg.norm(h1 - o) / np.linalg.norm(h2 - o)
        assert abs(np.degrees(np.arccos(cosang)) - 104.52) < 1e-6
