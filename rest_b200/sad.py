"""REST's SAD initial guess: superposition of atomic densities.

REST (src/initial_guess/sad.rs:8-117) runs, once per element of the molecule,
an SCF of the neutral atom in the molecule's basis and auxiliary basis, from the
hcore guess, unrestricted with the multiplicity of ctrl_setting_atom_sad
(:140-150: H, B, F and their groups doublets, C and O triplets, N quartets,
other elements closed-shell restricted, whose density is split in equal alpha
and beta halves), and places the atoms' alpha and beta densities on the
block diagonal of the molecule's AO order.  A restricted molecule starts from
alpha + beta.  The SCF driver then builds a Fock matrix from that density
(dm-only exchange), diagonalises it and takes the density of its orbitals as
the first input (initial_guess/mod.rs:46-58).

The atomic SCFs here run through rest_b200.scf.SCF on the device J/K, so
each atom's density is the same FP64 RI-HF density REST computes for it.  They
are cached per (element, basis, auxiliary basis) for the process.
"""
from __future__ import annotations

import numpy as np

from .basis import Molecule

# ctrl_setting_atom_sad (src/initial_guess/sad.rs:140-150): REST's `spin` keyword
# (the multiplicity) of each element's atomic SCF
_SPIN = {}
for _els, _m in ((("H", "Li", "Na", "K", "Rb", "Cs", "Fr"), 2), (("B", "Al", "Ga", "In", "Tl", "Nh"), 2),
                 (("C", "Si", "Ge", "Sn", "Pb", "Fl"), 3), (("N", "P", "As", "Sb", "Bi", "Mc"), 4),
                 (("O", "S", "Se", "Te", "Po", "Lv"), 3), (("F", "Cl", "Br", "I", "At", "Ts"), 2)):
    for _e in _els:
        _SPIN[_e] = _m

_CACHE: dict = {}


def atom_multiplicity(symbol: str) -> int:
    return _SPIN.get(symbol, 1)


def atom_densities(symbol: str, basis: str, auxbas: str, make_ctx=None) -> tuple[np.ndarray, np.ndarray]:
    """(alpha, beta) density of the neutral atom's SCF (cached).  make_ctx()
    gives the J/K context the atomic SCF loads its tensor into (default: a new
    device context on device 0), closed afterwards when it can be."""
    key = (symbol, basis, auxbas)
    if key not in _CACHE:
        from .rijk import RIJK
        from .scf import SCF, ScfOptions

        mol = Molecule.from_angstrom([symbol], [[0.0, 0.0, 0.0]], charge=0, spin=atom_multiplicity(symbol))
        ctx = make_ctx() if make_ctx is not None else RIJK(0)
        try:
            r = SCF(mol, basis, auxbas, ScfOptions(initial_guess="hcore"), ctx=ctx).run()
        finally:
            if hasattr(ctx, "close"):
                ctx.close()
        if not r.converged:
            raise RuntimeError(f"atomic SCF of {symbol} in {basis} did not converge")
        if len(r.density) == 1 or mol.spin == 1:
            half = 0.5 * np.asarray(r.density[0])
            _CACHE[key] = (half, half.copy())
        else:
            _CACHE[key] = (np.asarray(r.density[0]), np.asarray(r.density[1]))
    return _CACHE[key]


def sad_density(mol: Molecule, basis: str, auxbas: str, make_ctx=None) -> list:
    """The SAD density of ``mol``: [alpha + beta] for a restricted molecule
    (multiplicity 1), else [alpha, beta]; n x n each, the molecule's AO order
    (the shells of rest_b200.basis are atom by atom)."""
    sh = mol.shells(basis)
    n = sh.nfun
    da, db = np.zeros((n, n)), np.zeros((n, n))
    nf = 2 * sh.l + 1
    start = np.concatenate([[0], np.cumsum(nf)])
    for ia, sym in enumerate(mol.symbols):
        idx = np.nonzero(sh.atom == ia)[0]
        f0, f1 = int(start[idx[0]]), int(start[idx[-1] + 1])
        a, b = atom_densities(sym, basis, auxbas, make_ctx)
        if a.shape != (f1 - f0, f1 - f0):
            raise ValueError(f"atomic density of {sym} does not match its {f1 - f0} functions")
        da[f0:f1, f0:f1] = a
        db[f0:f1, f0:f1] = b
    return [da + db] if mol.spin == 1 else [da, db]
