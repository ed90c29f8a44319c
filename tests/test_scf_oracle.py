"""CPU pins of the integral engine and the SCF driver against REST's published run.

REST's example `examples/PEN/RIHF` (pentacene, STO-3G / def2-SV(P)-JKFIT, RI-HF)
printed its nuclear repulsion, lowest overlap eigenvalue, basis sizes and
converged energy; tests/golden/pen_rihf.json holds them.  The SCF loop of
rest_b200.scf runs here on the CPU oracle (oracle/scf_ctx.py).
"""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import rijk_oracle as O
from oracle.scf_ctx import OracleRIJK
from rest_b200.basis import Molecule, int1e, int2c2e, int3c2e, solid_harmonic_c2s
from rest_b200.scf import SCF, ScfOptions

GOLDEN = Path(__file__).resolve().parent / "golden"


def _pen():
    g = json.loads((GOLDEN / "pen_rihf.json").read_text())
    return g, Molecule.from_angstrom(g["symbols"], g["coords_angstrom"])


def test_h2_sto3g_textbook_integrals():
    """Szabo & Ostlund table 3.5 (H2, R = 1.4 bohr, STO-3G)."""
    mol = Molecule(["H", "H"], np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 1.4]]))
    sh = mol.shells("STO-3G")
    s = int1e(mol, sh, "ovlp")
    t = int1e(mol, sh, "kinetic")
    v = int1e(mol, sh, "nuclear")
    assert abs(s[0, 1] - 0.6593) < 1e-4
    assert abs(t[0, 0] - 0.7600) < 1e-4 and abs(t[0, 1] - 0.2365) < 1e-4
    assert abs(v[0, 0] + 1.8804) < 1e-4 and abs(v[0, 1] + 1.1948) < 1e-4


def test_solid_harmonics_are_orthonormal_on_the_sphere():
    from rest_b200.basis import _sphere_monomial, cart_components

    for l in range(5):
        c = solid_harmonic_c2s(l)
        comps = cart_components(l)
        g = np.array([[_sphere_monomial(a[0] + b[0], a[1] + b[1], a[2] + b[2]) for b in comps] for a in comps])
        assert np.allclose(c @ g @ c.T, np.eye(2 * l + 1), atol=1e-12)


def test_coulomb_integrals_are_rotation_invariant():
    """Eigenvalues of (P|Q) and of the three-centre Gram matrix do not change
    under a rigid rotation of the molecule (checks every l up to g)."""
    sy = ["O", "H", "H"]
    xyz = np.array([[0.0, 0.0, 0.1], [1.43, 1.1, 0.0], [-1.43, 1.1, 0.2]])
    rng = np.random.default_rng(0)
    q = np.linalg.qr(rng.standard_normal((3, 3)))[0]
    vals = []
    for r in (xyz, xyz @ q.T):
        mol = Molecule(sy, r)
        aux = mol.shells("def2-SVP-JKFIT")
        bas = mol.shells("def2-SVP")
        v2 = int2c2e(aux)
        i3 = int3c2e(bas, aux)
        # singular values of the full (n*n, N) tensor (the packed triangle is not
        # an orthogonal image of it, so only the unpacked form is invariant)
        full = O.ri3fn_from_rimatr(i3, bas.nfun).reshape(bas.nfun ** 2, aux.nfun, order="F")
        vals.append((np.linalg.eigvalsh(v2), np.linalg.svd(full, compute_uv=False)))
    assert np.allclose(vals[0][0], vals[1][0], rtol=1e-10, atol=1e-10)
    assert np.allclose(vals[0][1], vals[1][1], rtol=1e-10, atol=1e-10)


def test_pen_geometry_and_basis_match_rest():
    g, mol = _pen()
    assert abs(mol.nuclear_repulsion() - g["rest_nuc_energy"]) < 1e-9
    bas = mol.shells(g["basis"])
    aux = mol.shells(g["auxbas"])
    assert bas.nfun == g["rest_num_basis"] and aux.nfun == g["rest_num_auxbas"]
    s = int1e(mol, bas, "ovlp")
    assert abs(np.linalg.eigvalsh(s)[0] - g["rest_ovlp_lowest_eigenvalue"]) < 5e-9  # REST prints 8 digits


def test_water_oracle_scf_reproduces_golden():
    g = json.loads((GOLDEN / "water_rihf.json").read_text())
    mol = Molecule.from_angstrom(g["symbols"], g["coords_angstrom"])
    opts = ScfOptions(scf_acc_etot=1e-11, scf_acc_rho=1e-8, scf_acc_eev=1e-8, max_scf_cycle=200)
    r = SCF(mol, g["basis"], g["auxbas"], opts, ctx=OracleRIJK()).run()
    assert r.converged and (r.num_basis, r.num_auxbas) == (24, 113)
    assert abs(r.energy - g["oracle_energy"]) < 1e-10


def test_pen_rihf_energy_matches_rest():
    """The whole chain (integrals, V^-1/2 fit, J/K, SCF) against REST's log: 1e-8 Eh."""
    g, mol = _pen()
    opts = ScfOptions(scf_acc_etot=1e-10, scf_acc_rho=1e-7, scf_acc_eev=1e-7, max_scf_cycle=150)
    r = SCF(mol, g["basis"], g["auxbas"], opts, ctx=OracleRIJK()).run()
    assert r.converged
    assert abs(r.energy - g["rest_energy"]) < 1e-8
    # PySCF uses a different Bohr radius (0.52917721092): its energy differs by ~6e-8
    assert abs(r.energy - g["pyscf_energy"]) < 2e-7


def test_nh3_dimer_cation_fixture_pins_the_oracle_to_rest():
    """(NH3)2+ RI-UHF in aug-cc-pV5Z (REST examples/RIHF-NH3-dimer): the basis
    sizes built here equal REST's (734 / 262), and the CPU oracle's SCF from the
    same input (run by tests/golden/make_golden.py, about four minutes) lands on
    REST's published energy -111.9434834841 Eh within 1e-9 Eh; PySCF's differs by
    5e-9 Eh (another Bohr radius)."""
    import json

    g = json.loads((GOLDEN / "nh3_dimer_cation_rihf.json").read_text())
    mol = Molecule.from_angstrom(g["symbols"], g["coords_angstrom"], charge=g["charge"], spin=g["spin"])
    assert (mol.shells(g["basis"]).nfun, mol.shells(g["auxbas"]).nfun) == (g["rest_num_basis"], g["rest_num_auxbas"])
    assert mol.nelec == 19 and g["spin"] == 2
    assert abs(g["oracle_energy"] - g["rest_energy"]) < 1e-9
    assert abs(g["oracle_energy"] - g["pyscf_energy"]) < 2e-8


def test_density_difference_factor_is_exact():
    """The signed low-rank factor dD = V S V^T the mixed-precision SCF feeds to
    the split exchange build reproduces the density difference."""
    from rest_b200.scf import SCF

    rng = np.random.default_rng(4)
    n, o = 30, 6
    c1 = np.linalg.qr(rng.standard_normal((n, n)))[0]
    c2 = np.linalg.qr(c1 + 0.05 * rng.standard_normal((n, n)))[0]
    occ = np.zeros(n)
    occ[:o] = 2.0
    stub = SCF.__new__(SCF)
    stub.spin_channel, stub.n = 1, n
    t1 = stub.terms_of([c1], [occ], [o - 1])
    t2 = stub.terms_of([c2], [occ], [o - 1])
    for new, ref in ((t2, t1), (SCF.mix_terms(t1, t2, 0.6), t1)):
        d_new = sum(c * y @ y.T for c, y in new[0])
        d_ref = sum(c * y @ y.T for c, y in ref[0])
        v, npos = stub.delta_factor(new[0], ref[0])
        s = np.concatenate([np.ones(npos), -np.ones(v.shape[1] - npos)])
        assert np.max(np.abs((v * s) @ v.T - (d_new - d_ref))) < 1e-12
        assert v.shape[1] <= 4 * o


def test_sad_guess_matches_rest_recipe():
    """REST's SAD guess (src/initial_guess/sad.rs): neutral-atom UHF densities with
    the multiplicities of ctrl_setting_atom_sad (O triplet: 5 alpha + 3 beta
    electrons; H doublet), on the block diagonal; water from it reaches the same
    energy as from hcore in fewer iterations."""
    from rest_b200.sad import atom_densities, sad_density

    g = json.loads((GOLDEN / "water_rihf.json").read_text())
    mol = Molecule.from_angstrom(g["symbols"], g["coords_angstrom"])
    tight = dict(scf_acc_etot=1e-11, scf_acc_rho=1e-8, scf_acc_eev=1e-8, max_scf_cycle=200)
    r_h = SCF(mol, g["basis"], g["auxbas"], ScfOptions(initial_guess="hcore", **tight), ctx=OracleRIJK()).run()
    r_s = SCF(mol, g["basis"], g["auxbas"], ScfOptions(initial_guess="sad", **tight), ctx=OracleRIJK()).run()
    assert r_s.converged and abs(r_s.energy - g["oracle_energy"]) < 1e-9
    assert r_s.iterations < r_h.iterations
    for el, na, nb in (("O", 5, 3), ("H", 1, 0)):
        atom = Molecule.from_angstrom([el], [[0.0, 0.0, 0.0]])
        s = int1e(atom, atom.shells(g["basis"]), "ovlp")
        a, b = atom_densities(el, g["basis"], g["auxbas"], OracleRIJK)
        assert abs(np.trace(a @ s) - na) < 1e-10 and abs(np.trace(b @ s) - nb) < 1e-10
    d = sad_density(mol, g["basis"], g["auxbas"], OracleRIJK)[0]
    s = int1e(mol, mol.shells(g["basis"]), "ovlp")
    assert abs(np.trace(d @ s) - 10.0) < 1e-10
