"""Molecules, contracted Gaussian basis sets and their integrals (host side).

This is the input side of REST's RI build: ``Molecule::build``
(src/molecule_io/mod.rs:153) collects the basis (``collect_basis`` :498),
normalises every contraction (``BasCell::basis_normalization``,
src/basis_io/mod.rs:242-341: primitives scaled by the radial norm, the
contracted function by its self-overlap), converts Angstrom to Bohr with
ANG = 0.5291772083 (src/constants/mod.rs:85), and calls libcint for the
one-electron, two-centre and three-centre integrals.  Here the integrals come
from the library's own McMurchie-Davidson engine (``rijk_int1e``,
``rijk_int2c2e``, ``rijk_int3c2e``); functions are real solid harmonics.
"""
from __future__ import annotations

import ctypes as C
import json
import math
from dataclasses import dataclass, field
from fractions import Fraction
from pathlib import Path

import numpy as np

from ._abi import RijkError, lib

ANG = 0.5291772083  # Bohr radius in Angstrom used by REST (src/constants/mod.rs:85)
DATA = Path(__file__).resolve().parent / "basis_data"
Z_OF = {"H": 1, "He": 2, "Li": 3, "Be": 4, "B": 5, "C": 6, "N": 7, "O": 8, "F": 9, "Ne": 10, "Cu": 29}
LMAX = 6


# ---------------------------------------------------------------------------
# real solid harmonics
# ---------------------------------------------------------------------------
def cart_components(l: int):
    """(i, j, k) exponents, ordered by descending i then descending j."""
    return [(i, j, l - i - j) for i in range(l, -1, -1) for j in range(l - i, -1, -1)]


def _sphere_monomial(a: int, b: int, c: int) -> float:
    """Integral of x^a y^b z^c over the unit sphere."""
    if a % 2 or b % 2 or c % 2:
        return 0.0
    g = math.gamma
    return 2.0 * g((a + 1) / 2) * g((b + 1) / 2) * g((c + 1) / 2) / g((a + b + c + 3) / 2)


def solid_harmonic_c2s(l: int) -> np.ndarray:
    """(2l+1) x ncart matrix: rows are real solid harmonics S_lm, m = -l..l,
    expanded in Cartesian monomials (closed form of the expansion, e.g.
    Helgaker, Joergensen & Olsen, Molecular Electronic-Structure Theory, eq. 6.4.47),
    each row normalised on the unit sphere."""
    comps = cart_components(l)
    index = {c: n for n, c in enumerate(comps)}
    rows = []
    for m in range(-l, l + 1):
        am = abs(m)
        vm2 = 0 if m >= 0 else 1  # 2 * v_m
        coef = {}
        for t in range((l - am) // 2 + 1):
            for u in range(t + 1):
                # v = vm2/2, vm2/2 + 1, ..., up to floor(|m|/2 - v_m) + v_m
                v2 = vm2
                vmax2 = 2 * ((am - vm2) // 2) + vm2
                while v2 <= vmax2:
                    sign = -1 if ((t + (v2 - vm2) // 2) % 2) else 1
                    cval = (sign * Fraction(1, 4 ** t) * math.comb(l, t) * math.comb(l - t, am + t)
                            * math.comb(t, u) * math.comb(am, v2))
                    px = 2 * t + am - 2 * u - v2
                    py = 2 * u + v2
                    pz = l - 2 * t - am
                    key = (px, py, pz)
                    coef[key] = coef.get(key, 0) + cval
                    v2 += 2
        row = np.zeros(len(comps))
        for key, cval in coef.items():
            row[index[key]] += float(cval)
        # normalise on the unit sphere
        n2 = 0.0
        for a, ca in enumerate(comps):
            for b, cb in enumerate(comps):
                if row[a] and row[b]:
                    n2 += row[a] * row[b] * _sphere_monomial(ca[0] + cb[0], ca[1] + cb[1], ca[2] + cb[2])
        rows.append(row / math.sqrt(n2))
    return np.array(rows)


_C2S = [np.ascontiguousarray(solid_harmonic_c2s(l)) for l in range(LMAX + 1)]
_C2S_PTRS = (C.POINTER(C.c_double) * (LMAX + 1))(*[m.ctypes.data_as(C.POINTER(C.c_double)) for m in _C2S])


# ---------------------------------------------------------------------------
# basis sets and molecules
# ---------------------------------------------------------------------------
def load_basis(name: str) -> dict:
    f = DATA / f"{name}.json"
    if not f.exists():
        raise FileNotFoundError(f"basis {name!r} is not bundled ({f})")
    return json.loads(f.read_text())


def _radial_norm(l: int, a: float) -> float:
    """1 / sqrt(int_0^inf r^(2l+2) exp(-2 a r^2) dr) for a primitive r^l exp(-a r^2)."""
    return 1.0 / math.sqrt(math.gamma(l + 1.5) / (2.0 * (2.0 * a) ** (l + 1.5)))


def _contraction_norm(l: int, exps, coefs) -> float:
    s = 0.0
    for a, ca in zip(exps, coefs):
        for b, cb in zip(exps, coefs):
            s += ca * cb * _radial_norm(l, a) * _radial_norm(l, b) * math.gamma(l + 1.5) / (2.0 * (a + b) ** (l + 1.5))
    return 1.0 / math.sqrt(s)


@dataclass
class ShellSet:
    """Contracted shells of one basis on one molecule, as rijk_shells arrays."""
    l: np.ndarray
    nprim: np.ndarray
    prim_off: np.ndarray
    exps: np.ndarray
    coefs: np.ndarray
    centers: np.ndarray
    atom: np.ndarray
    _struct: object = field(default=None, repr=False)

    @property
    def nshell(self) -> int:
        return int(self.l.size)

    @property
    def nfun(self) -> int:
        return int(np.sum(2 * self.l + 1))

    def cstruct(self):
        from ._abi import RijkShells

        if self._struct is None:
            self._struct = RijkShells(
                self.nshell,
                self.l.ctypes.data_as(C.POINTER(C.c_int32)),
                self.nprim.ctypes.data_as(C.POINTER(C.c_int32)),
                self.prim_off.ctypes.data_as(C.POINTER(C.c_int64)),
                self.exps.ctypes.data_as(C.POINTER(C.c_double)),
                self.coefs.ctypes.data_as(C.POINTER(C.c_double)),
                self.centers.ctypes.data_as(C.POINTER(C.c_double)),
            )
        return self._struct


@dataclass
class Molecule:
    symbols: list
    coords: np.ndarray  # bohr, (natom, 3)
    charge: int = 0
    spin: int = 1  # multiplicity, as REST's `spin` keyword

    @staticmethod
    def from_angstrom(symbols, coords_ang, charge: int = 0, spin: int = 1) -> "Molecule":
        return Molecule(list(symbols), np.asarray(coords_ang, dtype=np.float64) / ANG, charge, spin)

    @property
    def charges(self) -> np.ndarray:
        return np.array([float(Z_OF[s]) for s in self.symbols])

    @property
    def nelec(self) -> int:
        return int(round(self.charges.sum())) - self.charge

    def nuclear_repulsion(self) -> float:
        """``calc_nuc_energy`` (src/geom_io/mod.rs:163-179)."""
        z, r = self.charges, self.coords
        e = 0.0
        for i in range(len(z)):
            for j in range(i):
                e += z[i] * z[j] / float(np.linalg.norm(r[i] - r[j]))
        return e

    def shells(self, basis: str) -> ShellSet:
        """The molecule's shells in ``basis`` (built once per basis and cached;
        the molecule's geometry is not meant to change after construction)."""
        cache = self.__dict__.setdefault("_shell_cache", {})
        if basis not in cache:
            cache[basis] = self._build_shells(basis)
        return cache[basis]

    def _build_shells(self, basis: str) -> ShellSet:
        data = load_basis(basis)
        ls, nps, offs, exps, coefs, ctrs, atoms = [], [], [], [], [], [], []
        off = 0
        for ia, (sym, xyz) in enumerate(zip(self.symbols, self.coords)):
            if sym not in data:
                raise KeyError(f"element {sym} is not in basis {basis}")
            for sh in data[sym]:
                l, e, c = sh["l"], sh["exps"], sh["coefs"]
                if l > LMAX:
                    raise ValueError(f"l = {l} above the supported {LMAX}")
                nc = _contraction_norm(l, e, c)
                ls.append(l)
                nps.append(len(e))
                offs.append(off)
                off += len(e)
                exps.extend(e)
                coefs.extend(ci * _radial_norm(l, ei) * nc for ei, ci in zip(e, c))
                ctrs.append(xyz)
                atoms.append(ia)
        return ShellSet(np.array(ls, dtype=np.int32), np.array(nps, dtype=np.int32), np.array(offs, dtype=np.int64),
                        np.array(exps, dtype=np.float64), np.array(coefs, dtype=np.float64),
                        np.ascontiguousarray(np.array(ctrs, dtype=np.float64)), np.array(atoms, dtype=np.int64))


# ---------------------------------------------------------------------------
# integrals
# ---------------------------------------------------------------------------
def _check(st: int, what: str):
    if st != 0:
        raise RijkError(st, what)


def int1e(mol: Molecule, sh: ShellSet, kind: str) -> np.ndarray:
    k = {"ovlp": 0, "kinetic": 1, "nuclear": 2}[kind]
    n = sh.nfun
    out = np.zeros((n, n), order="F")
    z = np.ascontiguousarray(mol.charges)
    xyz = np.ascontiguousarray(mol.coords)
    _check(lib().rijk_int1e(C.byref(sh.cstruct()), _C2S_PTRS, k, len(z), z.ctypes.data_as(C.POINTER(C.c_double)),
                            xyz.ctypes.data_as(C.POINTER(C.c_double)), out.ctypes.data_as(C.POINTER(C.c_double))),
           "int1e")
    return out


def int2c2e(aux: ShellSet) -> np.ndarray:
    n = aux.nfun
    out = np.zeros((n, n), order="F")
    _check(lib().rijk_int2c2e(C.byref(aux.cstruct()), _C2S_PTRS, out.ctypes.data_as(C.POINTER(C.c_double))),
           "int2c2e")
    return out


def int3c2e(bas: ShellSet, aux: ShellSet) -> np.ndarray:
    """(mu nu|P) in REST's rimatr layout [npair, naux] (Fortran order)."""
    n, naux = bas.nfun, aux.nfun
    out = np.zeros((n * (n + 1) // 2, naux), order="F")
    _check(lib().rijk_int3c2e(C.byref(bas.cstruct()), C.byref(aux.cstruct()), _C2S_PTRS,
                              out.ctypes.data_as(C.POINTER(C.c_double))), "int3c2e")
    return out


# angular-momentum limits of the device integral engine (rijk_int*_dev)
DEVICE_MAX_L_AO = 2
DEVICE_MAX_L_AUX = 4


def int2c2e_dev(aux: ShellSet, stream=None):
    """(P|Q) computed on the current CUDA device: a torch float64 tensor
    (naux, naux) whose storage is column-major (it is symmetric)."""
    import torch

    n = aux.nfun
    out = torch.empty((n, n), dtype=torch.float64, device="cuda")
    st = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    _check(lib().rijk_int2c2e_dev(C.byref(aux.cstruct()), _C2S_PTRS, C.c_void_p(out.data_ptr()), C.c_void_p(st)),
           "int2c2e_dev")
    return out


def int3c2e_dev(bas: ShellSet, aux: ShellSet, stream=None):
    """(mu nu|P) computed on the current CUDA device in rimatr layout: a torch
    float64 tensor of shape (naux, npair), row P = packed upper triangle of (..|P)."""
    import torch

    n, naux = bas.nfun, aux.nfun
    out = torch.empty((naux, n * (n + 1) // 2), dtype=torch.float64, device="cuda")
    st = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    _check(lib().rijk_int3c2e_dev(C.byref(bas.cstruct()), C.byref(aux.cstruct()), _C2S_PTRS,
                                  C.c_void_p(out.data_ptr()), C.c_void_p(st)), "int3c2e_dev")
    return out


# A nucleus as an s Gaussian of this exponent, normalised to its charge, is a
# point charge to double precision: in the three-centre kernel the product
# exponent p g / (p + g) evaluates to p because p + g rounds to g.
POINT_CHARGE_EXPONENT = 1.0e20


def point_charges(mol: Molecule) -> ShellSet:
    """The nuclei as auxiliary s shells carrying -Z (divided by the l = 0 solid
    harmonic factor that the three-centre engine applies)."""
    z = np.asarray(mol.charges, dtype=np.float64)
    na = len(z)
    g = POINT_CHARGE_EXPONENT
    coef = -z * (g / np.pi) ** 1.5 / _C2S[0][0, 0]
    return ShellSet(np.zeros(na, dtype=np.int32), np.ones(na, dtype=np.int32), np.arange(na, dtype=np.int64),
                    np.full(na, g), np.ascontiguousarray(coef), np.ascontiguousarray(mol.coords, dtype=np.float64),
                    np.arange(na, dtype=np.int64))


def int1e_nuclear_dev(mol: Molecule, sh: ShellSet, stream=None):
    """Nuclear attraction sum_C -Z_C (mu|1/|r - C||nu) on the current CUDA device,
    as the three-centre integrals with point charges summed over the nuclei: a
    torch float64 (n, n) tensor (the host engine's int1e(..., "nuclear"))."""
    import torch

    n = sh.nfun
    v = int3c2e_dev(sh, point_charges(mol), stream).sum(dim=0)  # packed upper, (i <= j) at j(j+1)/2 + i
    tri = torch.tril_indices(n, n, device=v.device)
    out = torch.zeros((n, n), dtype=torch.float64, device=v.device)
    out[tri[1], tri[0]] = v
    out[tri[0], tri[1]] = v
    return out
