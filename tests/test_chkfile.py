"""REST's HDF5 guess and checkpoint files (rest_b200.chkfile), on the CPU.

* Reader against libhdf5: tests/golden/cu2_init_guess.chk is REST's own
  example file (examples/Cu2/HF_SAD, written by libhdf5 through PySCF).  Its
  orbitals must be orthonormal under this library's def2-SVP overlap of Cu2
  (s to f shells) once the AO-order map is applied, its converged density and
  its SAD ``init_guess`` density must hold 58 electrons, and the converged
  density must be idempotent (D S D = 2 D).
* Writer: the files it makes have the superblock, root group and symbol-table
  structure libhdf5 wrote in that file, and read back bit for bit, one and two
  spins, for init_guess (src/initial_guess/mod.rs:71-83) and the chkfile
  (:85-124) as REST reads them.
"""
import hashlib
import json
import struct
from pathlib import Path

import numpy as np
import pytest

from rest_b200 import chkfile as H
from rest_b200.basis import Molecule, int1e

GOLDEN = Path(__file__).resolve().parent / "golden"
CU2 = GOLDEN / "cu2_init_guess.chk"


@pytest.fixture(scope="module")
def cu2():
    g = json.loads((GOLDEN / "cu2_chk.json").read_text())
    assert hashlib.sha256(CU2.read_bytes()).hexdigest() == g["sha256"]
    mol = Molecule.from_angstrom(g["symbols"], g["coords_angstrom"])
    bas = mol.shells(g["basis"])
    assert bas.nfun == g["num_basis"] and mol.nelec == g["nelec"]
    return g, bas, int1e(mol, bas, "ovlp")


def test_reader_lists_the_libhdf5_file(cu2):
    r = H.H5Reader.open(CU2)
    assert r.keys("/") == ["init_guess", "mol", "scf"]
    assert r.keys("/scf") == ["e_tot", "mo_coeff", "mo_energy", "mo_occ"]
    assert r.dataset("scf/e_tot").shape == ()
    assert r.dataset("scf/mo_coeff").shape == (62, 62)
    assert r.dataset("init_guess").shape == (62, 62)
    with pytest.raises(H.HDF5FormatError):
        r.dataset("mol")  # a string dataset: not a numeric type this reader takes


def test_rest_orbitals_are_orthonormal_under_this_overlap(cu2):
    g, bas, s = cu2
    e_tot, vecs, vals = H.read_chkfile(CU2, 62, 62, 1, shells=bas)
    c = vecs[0]
    assert np.isfinite(e_tot) and e_tot < -3000
    assert np.max(np.abs(c.T @ s @ c - np.eye(62))) < 1e-7
    assert np.all(np.diff(vals[0]) >= 0)  # orbital energies ascending
    occ = H.H5Reader.open(CU2).dataset("scf/mo_occ")
    d = (c * occ) @ c.T
    assert abs(np.trace(d @ s) - g["nelec"]) < 1e-6
    assert np.max(np.abs(d @ s @ d - 2.0 * d)) < 1e-7
    # without the AO-order map the p shells do not line up
    _, raw, _ = H.read_chkfile(CU2, 62, 62, 1)
    assert np.max(np.abs(raw[0].T @ s @ raw[0] - np.eye(62))) > 0.1


def test_rest_init_guess_density(cu2):
    g, bas, s = cu2
    d = H.read_init_guess(CU2, 62, 1, shells=bas)[0]
    assert np.array_equal(d, d.T)
    assert abs(np.trace(d @ s) - g["nelec"]) < 1e-9


def test_ao_order_map_is_a_permutation(cu2):
    _, bas, _ = cu2
    perm = H.rest_ao_order(bas)
    assert sorted(perm) == list(range(62))
    # the first p shell of Cu (functions 5, 6, 7 here: y, z, x) -> REST (x, y, z)
    assert list(perm[5:8]) == [7, 5, 6]


def _superblock(b: bytes):
    return struct.unpack_from("<8B HHI QQQQ", b, 8)


def test_writer_layout_matches_libhdf5(tmp_path, cu2):
    """Superblock fields, root symbol-table entry and root group B-tree / heap
    placement equal those of the libhdf5-written file (file size and data
    addresses differ)."""
    ref = CU2.read_bytes()
    out = tmp_path / "g.chk"
    H.write_init_guess(out, [np.eye(62)])
    mine = out.read_bytes()
    assert mine[:8] == ref[:8]
    sr, sm = _superblock(ref), _superblock(mine)
    assert sr[:8] == sm[:8] and sr[8:11] == sm[8:11]  # versions, sizes, K values, flags
    assert sr[11] == sm[11] == 0 and sr[12] == sm[12] and sr[14] == sm[14]  # base, free space, driver
    assert sm[13] == len(mine)  # end-of-file address
    # root entry: object header at 96, cached B-tree at 136 and heap at 680
    assert struct.unpack_from("<QQIIQQ", mine, 56) == struct.unpack_from("<QQIIQQ", ref, 56)


@pytest.mark.parametrize("spin", [1, 2])
def test_init_guess_round_trip(tmp_path, cu2, spin):
    _, bas, _ = cu2
    rng = np.random.default_rng(spin)
    dms = []
    for _ in range(spin):
        a = rng.standard_normal((62, 62))
        dms.append(a + a.T)
    out = tmp_path / "g.chk"
    H.write_init_guess(out, dms, shells=bas)
    back = H.read_init_guess(out, 62, spin, shells=bas)
    for a, b in zip(dms, back):
        assert np.array_equal(a, b)
    # REST's raw layout: spin s at [s n^2, (s+1) n^2), column-major, REST's AO order
    raw = H.H5Reader.open(out).dataset("init_guess").ravel()
    perm = H.rest_ao_order(bas)
    for s in range(spin):
        blk = raw[s * 62 * 62:(s + 1) * 62 * 62].reshape(62, 62, order="F")
        assert np.array_equal(blk, dms[s][np.ix_(perm, perm)])


@pytest.mark.parametrize("spin", [1, 2])
def test_chkfile_round_trip(tmp_path, cu2, spin):
    _, bas, _ = cu2
    rng = np.random.default_rng(10 + spin)
    cs = [rng.standard_normal((62, 62)) for _ in range(spin)]
    es = [np.sort(rng.standard_normal(62)) for _ in range(spin)]
    out = tmp_path / "c.chk"
    H.write_chkfile(out, -3280.5, cs, es, [np.full(62, 1.0)] * spin, shells=bas)
    e_tot, vecs, vals = H.read_chkfile(out, 62, 62, spin, shells=bas)
    assert e_tot == -3280.5
    for a, b in zip(cs, vecs):
        assert np.array_equal(a, b)
    for a, b in zip(es, vals):
        assert np.array_equal(a, b)
    r = H.H5Reader.open(out)
    assert r.keys("/scf") == ["e_tot", "mo_coeff", "mo_energy", "mo_occ"]
    assert r.dataset("scf/e_tot").shape == ()
    assert r.dataset("scf/mo_coeff").shape == ((62, 62) if spin == 1 else (2, 62, 62))


def test_libhdf5_file_rewritten_reads_the_same(tmp_path):
    """Every numeric dataset of REST's file, written again by this writer, reads
    back identical to the original."""
    r = H.H5Reader.open(CU2)
    w = H.H5Writer()
    names = ["init_guess"] + ["scf/" + k for k in r.keys("/scf")]
    for nm in names:
        w.create_dataset(nm, r.dataset(nm))
    out = tmp_path / "re.chk"
    w.save(out)
    r2 = H.H5Reader.open(out)
    for nm in names:
        a, b = r.dataset(nm), r2.dataset(nm)
        assert a.shape == b.shape and np.array_equal(a, b)


def test_not_hdf5_is_rejected(tmp_path):
    p = tmp_path / "x.chk"
    p.write_bytes(b"not an hdf5 file at all")
    with pytest.raises(H.HDF5FormatError):
        H.H5Reader.open(p)
