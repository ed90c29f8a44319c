"""Synthetic molecule generators of the benchmark configurations (seeded).

* water clusters (H2O)_k: O atoms by rejection sampling in a cube of side
  3.1 k^(1/3) A with a minimum O-O distance of 2.7 A, each water at the gas-phase
  geometry (O-H 0.9572 A, H-O-H 104.52 deg) with a uniformly random orientation;
* linear alkanes C_nH_{2n+2}: all-trans zigzag backbone, C-C 1.54 A, C-H 1.09 A,
  ideal tetrahedral angles.
"""
from __future__ import annotations

import numpy as np

from .basis import Molecule

TETRA = np.arccos(-1.0 / 3.0)  # 109.47 deg


def water_cluster(k: int, seed: int) -> Molecule:
    rng = np.random.default_rng(seed)
    side = 3.1 * k ** (1.0 / 3.0)
    oxy = []
    while len(oxy) < k:
        p = rng.uniform(0.0, side, 3)
        if all(np.linalg.norm(p - q) >= 2.7 for q in oxy):
            oxy.append(p)
    r, ang = 0.9572, np.deg2rad(104.52)
    local = np.array([[0.0, 0.0, 0.0], [r * np.sin(ang / 2), r * np.cos(ang / 2), 0.0],
                      [-r * np.sin(ang / 2), r * np.cos(ang / 2), 0.0]])
    symbols, coords = [], []
    for o in oxy:
        q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        if np.linalg.det(q) < 0:
            q[:, 0] = -q[:, 0]
        for sym, x in zip(["O", "H", "H"], local @ q.T + o):
            symbols.append(sym)
            coords.append(x)
    return Molecule.from_angstrom(symbols, np.array(coords))


def water_cluster_set_spec(nmol: int, seed: int = 2024, kmax: int = 16) -> list:
    """(k, seed) of each cluster of the seeded molecule set: k uniform in
    1..kmax drawn from ``seed``, cluster i placed with seed 50000 + i."""
    ks = np.random.default_rng(seed).integers(1, kmax + 1, nmol)
    return [(int(k), 50000 + i) for i, k in enumerate(ks)]


def water_cluster_set(nmol: int, seed: int = 2024, kmax: int = 16) -> list:
    return [water_cluster(k, s) for k, s in water_cluster_set_spec(nmol, seed, kmax)]


def alkane_coords(nc: int, cc: float = 1.54, ch: float = 1.09):
    """(symbols, coords in A) of all-trans C_nH_{2n+2}.

    The backbone zigzags in the xy plane; carbon i has virtual neighbours at the
    zigzag positions i-1 and i+1 even at the chain ends.  Each carbon carries
    two hydrogens out of the plane, opposite the bisector of its two (real or
    virtual) C-C bonds, and each chain end one more hydrogen along the bond to
    its missing neighbour, so every carbon is an ideal tetrahedron."""
    half = TETRA / 2.0
    dx, dy = cc * np.sin(half), cc * np.cos(half)

    def cpos(i):
        return np.array([i * dx, (i % 2) * dy, 0.0])

    symbols, coords = [], []
    for i in range(nc):
        symbols.append("C")
        coords.append(cpos(i))
    z = np.array([0.0, 0.0, 1.0])
    for i in range(nc):
        c = cpos(i)
        u1 = cpos(i - 1) - c
        u2 = cpos(i + 1) - c
        u1 /= np.linalg.norm(u1)
        u2 /= np.linalg.norm(u2)
        b = -(u1 + u2)
        b /= np.linalg.norm(b)
        for sgn in (1.0, -1.0):
            symbols.append("H")
            coords.append(c + ch * (np.cos(half) * b + sgn * np.sin(half) * z))
        if i == 0:
            symbols.append("H")
            coords.append(c + ch * u1)
        if i == nc - 1:
            symbols.append("H")
            coords.append(c + ch * u2)
    return symbols, np.array(coords)


def alkane(nc: int) -> Molecule:
    symbols, coords = alkane_coords(nc)
    return Molecule.from_angstrom(symbols, coords)
