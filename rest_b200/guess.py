"""Learned initial guess: a per-atom-pair MLP that predicts AO density blocks.

For every ordered atom pair (A, B) closer than 6 A, the network maps features
of the pair and its surroundings to the density block D[AO(A), AO(B)] written
in the local frame of A's water molecule; the predicted blocks are rotated
back, symmetrised and assembled into the AO density that starts the SCF.

  frame       per water: origin O, axes p = unit(OH1 - OH2), b = unit(OH1 + OH2),
              n = p x b (rows of F); a block in the frame is G_A^T D_AB G_B with
              G_X the block-diagonal rotation of X's shells (real solid
              harmonics of l = 0, 1, 2 under r -> F^T r, from exact
              polynomial fits on sample points);
  features    element one-hots, B and B's water atoms in A's frame, A in its own
              frame, and Gaussian radial counts of O and H neighbours of A and of
              B (8 + 8 each, smooth 6 A cutoff): 53 numbers, standardised;
  network     53 -> 256 -> 256 -> 256 -> 256 -> 196 (SiLU), BF16 weights and
              activations with FP32 accumulation; output = the 14 x 14 block
              (O: 14 functions, H: 5 in def2-SVP; unused entries masked),
              standardised per element pair and entry;
  kernels     forward, backward, masked MSE and Adam are the library's own
              (rijk_mlp_*); at inference the frames, shell rotations, pairs and
              standardised features of a whole molecule set are built on the
              device (rijk_guess_geometry, rijk_guess_pairs) and the density is
              assembled there (rijk_guess_assemble); torch only holds the device
              memory (the host restatement below builds the training rows);
  fallback    a prediction whose electron count tr(D S) is off by more than 5 %
              (or not finite) is dropped for REST's own guess (hcore here).

REST has no learned guess: its guesses (src/initial_guess/mod.rs) are the fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from ._abi import RijkError, lib
from .basis import ANG, cart_components, solid_harmonic_c2s

CUTOFF = 6.0  # A
NFEAT = 53
BLOCK = 14
HIDDEN = 256
LAYERS = [NFEAT, HIDDEN, HIDDEN, HIDDEN, HIDDEN, BLOCK * BLOCK]
ELEMENT = {"O": 0, "H": 1}
RAD_MU = np.linspace(1.0, 6.0, 8)
RAD_SIGMA = 0.5
DEFAULT_WEIGHTS = Path(__file__).resolve().parent / "data" / "guess_h2o_def2svp.npz"


# ---------------------------------------------------------------------------
# geometry: frames, shell rotations, atom blocks
# ---------------------------------------------------------------------------
_C2S = {}  # l -> (Cartesian exponents, solid_harmonic_c2s(l)^T): exact-fraction expansion, built once


def _harmonics(l: int, u: np.ndarray) -> np.ndarray:
    """Real solid harmonics of degree l at points u (S x 3): S x (2l+1)."""
    if l not in _C2S:
        _C2S[l] = (cart_components(l), np.ascontiguousarray(solid_harmonic_c2s(l).T))
    comps, c2s_t = _C2S[l]
    mono = np.stack([u[:, 0] ** i * u[:, 1] ** j * u[:, 2] ** k for i, j, k in comps], axis=1)
    return mono @ c2s_t


_SAMPLES = np.random.default_rng(12345).standard_normal((40, 3))


def shell_rotation(l: int, F: np.ndarray) -> np.ndarray:
    """G with Y_l(F^T u) = G Y_l(u) for all u (exact: both sides are degree-l
    harmonic polynomials, fitted on 40 points)."""
    if l == 0:
        return np.ones((1, 1))
    y_loc = _harmonics(l, _SAMPLES)
    y_rot = _harmonics(l, _SAMPLES @ F)  # rows: F^T u_s
    gt, *_ = np.linalg.lstsq(y_loc, y_rot, rcond=None)
    return gt.T


@dataclass
class Frames:
    xyz: np.ndarray  # (na, 3) coordinates in A; water w's origin is its O, xyz[3 w]
    F: np.ndarray  # (nw, 3, 3) each water's frame, axes as rows


def water_frames(mol) -> Frames:
    """Per water (atoms 3w, 3w+1, 3w+2 = O, H1, H2): its frame F (rows), all
    waters at once; the frame's origin is the water's O."""
    xyz = np.asarray(mol.coords, dtype=np.float64) * ANG
    nw = len(mol.symbols) // 3
    if list(mol.symbols) != ["O", "H", "H"] * nw:
        raise ValueError("the learned guess is trained on water clusters (atoms ordered O, H, H per water)")
    w = xyz.reshape(nw, 3, 3)
    h1, h2 = w[:, 1] - w[:, 0], w[:, 2] - w[:, 0]
    p = h1 - h2
    b = h1 + h2
    p = p / np.linalg.norm(p, axis=1, keepdims=True)
    b = b - np.sum(b * p, axis=1, keepdims=True) * p
    b = b / np.linalg.norm(b, axis=1, keepdims=True)
    n = np.stack([p[:, 1] * b[:, 2] - p[:, 2] * b[:, 1], p[:, 2] * b[:, 0] - p[:, 0] * b[:, 2],
                  p[:, 0] * b[:, 1] - p[:, 1] * b[:, 0]], axis=1)
    return Frames(xyz, np.stack([p, b, n], axis=1))


def atom_layout(sh):
    """Per atom: (first AO, number of AOs, tuple of shell l)."""
    layout = {}
    off = 0
    for l, a in zip(sh.l, sh.atom):
        a = int(a)
        if a not in layout:
            layout[a] = [off, 0, []]
        if layout[a][0] + layout[a][1] != off:
            raise ValueError("shells of an atom must be contiguous")
        layout[a][1] += 2 * int(l) + 1
        layout[a][2].append(int(l))
        off += 2 * int(l) + 1
    return {a: (v[0], v[1], tuple(v[2])) for a, v in layout.items()}


def atom_rotation(shell_ls, rots) -> np.ndarray:
    n = sum(2 * l + 1 for l in shell_ls)
    g = np.zeros((n, n))
    o = 0
    for l in shell_ls:
        g[o:o + 2 * l + 1, o:o + 2 * l + 1] = rots[l]
        o += 2 * l + 1
    return g


def _radial(d: np.ndarray) -> np.ndarray:
    """Gaussian radial counts with a smooth cutoff: d (...,) -> (..., 8)."""
    fc = np.where(d < CUTOFF, 0.5 * (np.cos(np.pi * d / CUTOFF) + 1.0), 0.0)
    return np.exp(-((d[..., None] - RAD_MU) ** 2) / RAD_SIGMA ** 2) * fc[..., None]


@dataclass
class PairSet:
    feats: np.ndarray  # (P, NFEAT)
    pairs: np.ndarray  # (P, 2) atom indices (A, B)
    kind: np.ndarray  # (P,) 2 * type(A) + type(B)


def pair_features(mol, frames: Frames | None = None) -> PairSet:
    fr = frames if frames is not None else water_frames(mol)
    xyz, Fs = fr.xyz, fr.F
    na = len(mol.symbols)
    typ = np.array([ELEMENT[s] for s in mol.symbols])
    d = np.linalg.norm(xyz[:, None] - xyz[None], axis=-1)
    rad = _radial(d) * (1.0 - np.eye(na))[:, :, None]  # no self term
    env = np.concatenate([rad[:, typ == 0].sum(axis=1), rad[:, typ == 1].sum(axis=1)], axis=1)
    A, B = np.nonzero(d <= CUTOFF)
    wa, wb = A // 3, B // 3
    loc = np.matmul(xyz, np.transpose(Fs, (0, 2, 1)))  # (nw, na, 3): every atom in every water's axes
    la = loc[wa, A]
    db = loc[wa, B] - la
    wat = (loc[wa[:, None], 3 * wb[:, None] + np.arange(3)] - la[:, None, :]).reshape(len(A), 9)  # B's water
    own = la - loc[wa, 3 * wa]  # A relative to its own water's O (the frame origin)
    eye = np.eye(2)
    feats = np.concatenate([eye[typ[A]], eye[typ[B]], db, np.linalg.norm(db, axis=1)[:, None],
                            (wa == wb).astype(float)[:, None], wat, own, env[A], env[B]], axis=1)
    return PairSet(feats, np.stack([A, B], axis=1), 2 * typ[A] + typ[B])


class Rotator:
    """Per water w and element: G(F_w), the rotation of that element's AO block
    into the water's frame (every atom of an element has the same shells)."""

    def __init__(self, mol, sh, frames: Frames | None = None):
        Fs = (frames if frames is not None else water_frames(mol)).F
        self.layout = atom_layout(sh)
        typ = np.array([ELEMENT[s] for s in mol.symbols])
        self.typ = typ
        self.first = np.array([self.layout[a][0] for a in range(len(typ))])
        self.size, self.rot = {}, {}
        rots = {l: shell_rotations(l, Fs) for l in range(3)}
        for t in (0, 1):
            atoms = np.nonzero(typ == t)[0]
            if atoms.size == 0:
                continue
            shells = {self.layout[a][2] for a in atoms}
            if len(shells) != 1:
                raise ValueError("atoms of one element must carry the same shells")
            ls = shells.pop()
            self.size[t] = sum(2 * l + 1 for l in ls)
            g = np.zeros((len(Fs), self.size[t], self.size[t]))
            o = 0
            for l in ls:
                g[:, o:o + 2 * l + 1, o:o + 2 * l + 1] = rots[l]
                o += 2 * l + 1
            self.rot[t] = g

    def kinds(self, ps: PairSet):
        """(selection, rows (P,na), cols (P,nb), G_A (P,na,na), G_B (P,nb,nb)) per element pair."""
        for k in range(4):
            sel = np.nonzero(ps.kind == k)[0]
            if sel.size == 0:
                continue
            ta, tb = k // 2, k % 2
            a, b = ps.pairs[sel, 0], ps.pairs[sel, 1]
            w = a // 3
            rows = self.first[a][:, None] + np.arange(self.size[ta])
            cols = self.first[b][:, None] + np.arange(self.size[tb])
            yield sel, rows, cols, self.rot[ta][w], self.rot[tb][w]


_PINV = {}  # l -> pseudo-inverse of the harmonics at the sample points (a constant)


def shell_rotations(l: int, Fs: np.ndarray) -> np.ndarray:
    """shell_rotation for a stack of frames: (nw, 2l+1, 2l+1), all frames in one
    evaluation of the harmonics."""
    if l == 0:
        return np.ones((len(Fs), 1, 1))
    if l not in _PINV:
        _PINV[l] = np.linalg.pinv(_harmonics(l, _SAMPLES))
    pts = np.matmul(_SAMPLES, Fs).reshape(-1, 3)  # rows: F^T u_s for every frame
    y_rot = _harmonics(l, pts).reshape(len(Fs), len(_SAMPLES), 2 * l + 1)
    return np.transpose(_PINV[l] @ y_rot, (0, 2, 1))


def local_blocks(mol, sh, D: np.ndarray, ps: PairSet):
    """Targets: G_A^T D_AB G_B in A's water frame, padded to 14 x 14, with masks."""
    rot = Rotator(mol, sh)
    T = np.zeros((len(ps.pairs), BLOCK, BLOCK))
    M = np.zeros_like(T)
    for sel, rows, cols, ga, gb in rot.kinds(ps):
        blk = D[rows[:, :, None], cols[:, None, :]]
        T[sel, :rows.shape[1], :cols.shape[1]] = np.transpose(ga, (0, 2, 1)) @ blk @ gb
        M[sel, :rows.shape[1], :cols.shape[1]] = 1.0
    return T.reshape(len(ps.pairs), -1), M.reshape(len(ps.pairs), -1)


def assembly_inputs(mol, sh, ps: PairSet, rot: Rotator | None = None):
    """Host arrays of the device assembly (rijk_guess_assemble): unordered pairs
    (A, B, row of (A, B), row of (B, A)), per-atom first AO / type / AO count /
    water, and per water and element the 14 x 14 block rotation."""
    rot = rot if rot is not None else Rotator(mol, sh)
    na = len(mol.symbols)
    nw = na // 3
    R = np.zeros((nw, 2, BLOCK, BLOCK))
    for t, g in rot.rot.items():
        R[:, t, :g.shape[1], :g.shape[2]] = g
    first = np.array([rot.layout[a][0] for a in range(na)], dtype=np.int32)
    nfun = np.array([rot.layout[a][1] for a in range(na)], dtype=np.int32)
    A, B = ps.pairs[:, 0].astype(np.int64), ps.pairs[:, 1].astype(np.int64)
    key = A * na + B
    order = np.argsort(key)
    sel = np.nonzero(A <= B)[0]
    back = order[np.searchsorted(key[order], B[sel] * na + A[sel])]
    up = np.stack([A[sel], B[sel], sel, back], axis=1).astype(np.int32)
    return up, first, rot.typ.astype(np.int32), nfun, (np.arange(na) // 3).astype(np.int32), R


def assemble_density(mol, sh, ps: PairSet, blocks: np.ndarray) -> np.ndarray:
    """Rotate predicted local blocks back, D_AB = G_A B G_B^T, and average the
    (A, B) and (B, A)^T predictions; pairs beyond the cutoff stay zero."""
    rot = Rotator(mol, sh)
    n = sh.nfun
    D = np.zeros((n, n))
    cnt = np.zeros((n, n))
    blocks = blocks.reshape(len(ps.pairs), BLOCK, BLOCK)
    for sel, rows, cols, ga, gb in rot.kinds(ps):
        full = ga @ blocks[sel, :rows.shape[1], :cols.shape[1]] @ np.transpose(gb, (0, 2, 1))
        r, c = rows[:, :, None], cols[:, None, :]
        np.add.at(D, (r, c), full)
        np.add.at(cnt, (r, c), 1.0)
        np.add.at(D, (c.transpose(0, 2, 1), r.transpose(0, 2, 1)), np.transpose(full, (0, 2, 1)))
        np.add.at(cnt, (c.transpose(0, 2, 1), r.transpose(0, 2, 1)), 1.0)
    return D / np.maximum(cnt, 1.0)


# ---------------------------------------------------------------------------
# the network on the device (library kernels)
# ---------------------------------------------------------------------------
def _ck(st: int, what: str):
    if st != 0:
        raise RijkError(st, what)


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


_GEO_TABLE = []  # the constants of rijk_guess_geometry, built once


def geometry_table() -> np.ndarray:
    """The 516 constants of the device geometry (rijk_guess_geometry): the 40
    sample points; for l = 1, 2 the Cartesian exponents, the c2s expansion
    transposed and the pseudo-inverse of the harmonics at the samples (the fit
    shell_rotations makes); the cutoff, the radial width and the 8 centres."""
    if not _GEO_TABLE:
        parts = [_SAMPLES.ravel()]
        for l in (1, 2):
            if l not in _PINV:
                _PINV[l] = np.linalg.pinv(_harmonics(l, _SAMPLES))
            parts += [np.asarray(cart_components(l), dtype=np.float64).ravel(), solid_harmonic_c2s(l).T.ravel(),
                      _PINV[l].ravel()]
        parts += [np.array([CUTOFF, RAD_SIGMA]), RAD_MU]
        t = np.ascontiguousarray(np.concatenate(parts), dtype=np.float64)
        if t.size != 516:
            raise AssertionError("geometry table layout")
        _GEO_TABLE.append(t)
    return _GEO_TABLE[0]


@dataclass
class DevicePairs:
    """A molecule set's pair rows on the device (rijk_guess_geometry +
    rijk_guess_pairs): standardised features (P x 53, FP32), unordered pairs
    (U x 4 int32, molecule-relative), per atom first AO / type / AO count / water
    (int32, molecule-relative), per water the block rotations; and on the host
    the offsets of each molecule's rows (nmol + 1 each) and its AO count."""
    feats: object
    up: object
    first: object
    typ: object
    nfun: object
    water: object
    rot: object
    pair_off: np.ndarray
    up_off: np.ndarray
    atom_off: np.ndarray
    nbas: np.ndarray


@dataclass
class PairLayout:
    """Host side of device_pairs: coordinates (A) and per-atom layout of a set
    of water clusters, molecule after molecule."""
    xyz: np.ndarray  # (natom, 3)
    info: np.ndarray  # (natom, 3) int32: first atom of the molecule, its atom count, element type
    first: np.ndarray  # (natom,) int32 first AO within the molecule
    typ: np.ndarray  # (natom,) int32 0 = O, 1 = H
    nfun: np.ndarray  # (natom,) int32 AO count
    water: np.ndarray  # (natom,) int32 water index within the molecule
    elem_shells: np.ndarray  # (2, 16) int32 per element: shell count, then each shell's l
    atom_off: np.ndarray  # (nmol + 1,) first atom of each molecule
    nbas: np.ndarray  # (nmol,) AO count of each molecule


def pair_layout(mols, basis: str) -> PairLayout:
    """The per-atom layout the geometry kernels take, vectorised over the set;
    every atom of an element carries that element's shells (one basis per
    element), checked against each molecule's AO count."""
    na = np.array([len(m.symbols) for m in mols], dtype=np.int64)
    for m in mols:
        if not m.symbols or list(m.symbols) != ["O", "H", "H"] * (len(m.symbols) // 3):
            raise ValueError("the learned guess is trained on water clusters (atoms ordered O, H, H per water)")
    atom_off = np.concatenate([[0], np.cumsum(na)])
    natom = int(atom_off[-1])
    if natom == 0:
        raise ValueError("empty molecule set")
    ref = mols[0].shells(basis)
    shells = {t: [int(l) for l in ref.l[ref.atom == t]] for t in (0, 1)}
    size = np.array([sum(2 * l + 1 for l in shells[t]) for t in (0, 1)], dtype=np.int64)
    if max(size) > BLOCK or any(l > 2 for t in (0, 1) for l in shells[t]) or any(len(v) > 15 for v in shells.values()):
        raise ValueError("the learned guess covers blocks of at most 14 functions with l <= 2")
    typ = np.tile(np.array([0, 1, 1], dtype=np.int32), natom // 3)
    nf = size[typ]
    csum = np.cumsum(nf)
    mstart = np.repeat(atom_off[:-1], na)
    first = (csum - nf - np.concatenate([[0], csum])[mstart]).astype(np.int32)
    nbas = np.add.reduceat(nf, atom_off[:-1]).astype(np.int64)
    for m, nb in zip(mols, nbas):
        sh = m.shells(basis)
        if sh.nfun != nb or np.any(np.diff(sh.atom) < 0):
            raise ValueError("shells of an atom must be contiguous and follow the element's basis")
    es = np.zeros((2, 16), dtype=np.int32)
    for t in (0, 1):
        es[t, 0] = len(shells[t])
        es[t, 1:1 + len(shells[t])] = shells[t]
    return PairLayout(xyz=np.concatenate([np.asarray(m.coords, dtype=np.float64) for m in mols]) * ANG,
                      info=np.stack([mstart, np.repeat(na, na), typ], axis=1).astype(np.int32), first=first, typ=typ,
                      nfun=nf.astype(np.int32), water=((np.arange(natom) - mstart) // 3).astype(np.int32),
                      elem_shells=es, atom_off=atom_off, nbas=nbas)


def device_pairs(mols, basis: str, norm: Normaliser, dev) -> DevicePairs:
    """The pair rows of a set of water clusters, built on the device; the host
    sends coordinates and the per-atom layout, and reads back one scan."""
    import torch

    lo = pair_layout(mols, basis)
    natom = len(lo.typ)
    atom_off, nbas = lo.atom_off, lo.nbas

    def dv(a, dtype):
        return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype).to(dev, non_blocking=False)

    x_d, info_d = dv(lo.xyz, torch.float64), dv(lo.info, torch.int32)
    tab_d, es_d = dv(geometry_table(), torch.float64), dv(lo.elem_shells, torch.int32)
    lay = dv(np.stack([lo.first, lo.typ, lo.nfun, lo.water]), torch.int32)  # rows: first, type, nfun, water
    nw = natom // 3
    frames = torch.empty(nw, 9, dtype=torch.float64, device=dev)
    rot = torch.empty(nw, 2, BLOCK, BLOCK, dtype=torch.float64, device=dev)
    counts = torch.empty(natom, 2, dtype=torch.int64, device=dev)
    env = torch.empty(natom, 16, dtype=torch.float64, device=dev)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    _ck(lib().rijk_guess_geometry(_p(x_d), _p(info_d), natom, _p(tab_d), _p(es_d), _p(frames), _p(rot), _p(counts),
                                  _p(env), stream), "guess_geometry")
    incl = torch.cumsum(counts, dim=0)
    excl = (incl - counts).t().contiguous()  # rows: pair offsets, unordered-pair offsets
    incl_h = incl.cpu().numpy()  # the one host read: each molecule's pair and unordered-pair rows
    start = np.concatenate([np.zeros((1, 2), dtype=np.int64), incl_h])[atom_off]
    npairs, nup = int(start[-1, 0]), int(start[-1, 1])
    feats = torch.empty(npairs, NFEAT, dtype=torch.float32, device=dev)
    up = torch.empty(nup, 4, dtype=torch.int32, device=dev)
    fm, fs = dv(norm.f_mean, torch.float64), dv(norm.f_std, torch.float64)
    _ck(lib().rijk_guess_pairs(_p(x_d), _p(info_d), natom, _p(tab_d), _p(frames), _p(env), _p(excl[0]),
                               _p(excl[1]), npairs, nup, _p(fm), _p(fs), _p(feats), _p(up), stream), "guess_pairs")
    return DevicePairs(feats, up, lay[0], lay[1], lay[2], lay[3], rot, start[:, 0], start[:, 1], atom_off, nbas)


class PairMLP:
    """MLP with FP32 master weights, BF16 working copies and Adam moments, all
    on the device; every step is a library kernel on torch's current stream."""

    def __init__(self, layers=LAYERS, seed: int = 0, device: int = 0):
        import torch

        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.layers = list(layers)
        rng = np.random.default_rng(seed)
        self.W, self.b, self.Wbf = [], [], []
        self.mW, self.vW, self.mb, self.vb = [], [], [], []
        for k, n in zip(self.layers[:-1], self.layers[1:]):
            lim = np.sqrt(6.0 / (k + n))
            w = torch.tensor(rng.uniform(-lim, lim, (n, k)), dtype=torch.float32, device=self.dev)
            self.W.append(w)
            self.b.append(torch.zeros(n, dtype=torch.float32, device=self.dev))
            self.Wbf.append(torch.empty(n, k, dtype=torch.int16, device=self.dev))
            for lst, shape in ((self.mW, (n, k)), (self.vW, (n, k)), (self.mb, (n,)), (self.vb, (n,))):
                lst.append(torch.zeros(shape, dtype=torch.float32, device=self.dev))
        self.step = 0
        self.sync_bf16()

    @property
    def stream(self):
        return C.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    def sync_bf16(self):
        for w, wb in zip(self.W, self.Wbf):
            _ck(lib().rijk_mlp_to_bf16(_p(w), _p(wb), w.numel(), self.stream), "to_bf16")

    def to_bf16(self, x):
        out = self.torch.empty(x.shape, dtype=self.torch.int16, device=self.dev)
        _ck(lib().rijk_mlp_to_bf16(_p(x), _p(out), x.numel(), self.stream), "to_bf16")
        return out

    def forward(self, xbf, keep: bool = False):
        """x (m x in, BF16 bits) -> y (m x out, FP32); keep=True also returns the
        per-layer inputs (BF16) and pre-activations for the backward pass."""
        torch = self.torch
        m = xbf.shape[0]
        h, acts, zs = xbf, [xbf], []
        nl = len(self.W)
        y = None
        for li, (wb, b) in enumerate(zip(self.Wbf, self.b)):
            n, k = wb.shape
            last = li == nl - 1
            z = torch.empty(m, n, dtype=torch.float32, device=self.dev) if keep else None
            if last:
                y = torch.empty(m, n, dtype=torch.float32, device=self.dev)
                _ck(lib().rijk_mlp_linear_fwd(_p(h), _p(wb), _p(b), m, k, n, 0, _p(z), None, _p(y), self.stream),
                    "linear_fwd")
            else:
                hn = torch.empty(m, n, dtype=torch.int16, device=self.dev)
                _ck(lib().rijk_mlp_linear_fwd(_p(h), _p(wb), _p(b), m, k, n, 1, _p(z), _p(hn), None, self.stream),
                    "linear_fwd")
                h = hn
                acts.append(h)
            zs.append(z)
        return (y, acts, zs) if keep else y

    def gradients(self, xbf, target, mask, norm: float):
        """Loss and per-layer (dW, db) of the masked MSE for one minibatch."""
        torch = self.torch
        y, acts, zs = self.forward(xbf, keep=True)
        m = xbf.shape[0]
        loss = torch.zeros(1, dtype=torch.float32, device=self.dev)
        dy = torch.empty_like(y)
        _ck(lib().rijk_mlp_masked_mse(_p(y), _p(target), _p(mask), y.numel(), float(norm), _p(dy), _p(loss),
                                      self.stream), "masked_mse")
        grads = [None] * len(self.W)
        for li in range(len(self.W) - 1, -1, -1):
            wb = self.Wbf[li]
            n, k = wb.shape
            dz = torch.empty(m, n, dtype=torch.int16, device=self.dev)
            dw = torch.empty(n, k, dtype=torch.float32, device=self.dev)
            db = torch.empty(n, dtype=torch.float32, device=self.dev)
            dx = torch.empty(m, k, dtype=torch.float32, device=self.dev) if li > 0 else None
            act = 0 if li == len(self.W) - 1 else 1
            _ck(lib().rijk_mlp_linear_bwd(_p(acts[li]), _p(wb), _p(zs[li]), _p(dy), m, k, n, act, _p(dz), _p(dw),
                                          _p(db), _p(dx), self.stream), "linear_bwd")
            grads[li] = (dw, db)
            dy = dx
        return loss, grads

    def adam_step(self, grads, lr: float, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step += 1
        for li, (dw, db) in enumerate(grads):
            _ck(lib().rijk_mlp_adam(_p(self.W[li]), _p(self.Wbf[li]), _p(dw), _p(self.mW[li]), _p(self.vW[li]),
                                    dw.numel(), lr, beta1, beta2, eps, self.step, self.stream), "adam")
            _ck(lib().rijk_mlp_adam(_p(self.b[li]), None, _p(db), _p(self.mb[li]), _p(self.vb[li]), db.numel(), lr,
                                    beta1, beta2, eps, self.step, self.stream), "adam")

    def state(self) -> dict:
        out = {}
        for i, (w, b) in enumerate(zip(self.W, self.b)):
            out[f"W{i}"] = w.cpu().numpy()
            out[f"b{i}"] = b.cpu().numpy()
        return out

    def load_state(self, st: dict):
        torch = self.torch
        for i in range(len(self.W)):
            self.W[i] = torch.tensor(st[f"W{i}"], dtype=torch.float32, device=self.dev)
            self.b[i] = torch.tensor(st[f"b{i}"], dtype=torch.float32, device=self.dev)
        self.sync_bf16()


# ---------------------------------------------------------------------------
# normalisation, training, prediction
# ---------------------------------------------------------------------------
@dataclass
class Normaliser:
    f_mean: np.ndarray
    f_std: np.ndarray
    t_mean: np.ndarray  # (4, 196) per element pair
    t_std: np.ndarray  # (4, 196)

    @staticmethod
    def fit(feats, targets, masks, kinds):
        t_mean = np.zeros((4, BLOCK * BLOCK))
        t_std = np.ones((4, BLOCK * BLOCK))
        for k in range(4):
            sel = kinds == k
            if sel.any():
                t_mean[k] = targets[sel].mean(axis=0)
                t_std[k] = np.maximum(targets[sel].std(axis=0), 1e-3) * masks[sel].max(axis=0) + \
                    (1.0 - masks[sel].max(axis=0))
        return Normaliser(feats.mean(axis=0), np.maximum(feats.std(axis=0), 1e-6), t_mean, t_std)

    def feats(self, f):
        return (f - self.f_mean) / self.f_std

    def targets(self, t, kinds):
        return (t - self.t_mean[kinds]) / self.t_std[kinds]

    def blocks(self, y, kinds):
        return y * self.t_std[kinds] + self.t_mean[kinds]


def training_arrays(samples, basis: str = "def2-SVP"):
    """samples: (molecule, converged density) pairs -> features, targets, masks, kinds."""
    F, T, M, K = [], [], [], []
    for mol, D in samples:
        sh = mol.shells(basis)
        ps = pair_features(mol)
        t, m = local_blocks(mol, sh, D, ps)
        F.append(ps.feats)
        T.append(t.astype(np.float32))  # the network trains in FP32 / BF16
        M.append(m.astype(np.float32))
        K.append(ps.kind)
    return np.concatenate(F), np.concatenate(T), np.concatenate(M), np.concatenate(K)


def train(samples, epochs: int = 60, batch: int = 4096, lr: float = 1e-3, seed: int = 0, basis: str = "def2-SVP",
          log=None):
    """Train the pair MLP on (molecule, converged FP64 density) samples on the device."""
    import torch

    feats, targets, masks, kinds = training_arrays(samples, basis)
    norm = Normaliser.fit(feats, targets, masks, kinds)
    net = PairMLP(seed=seed)
    dev = net.dev
    X = net.to_bf16(torch.tensor(norm.feats(feats), dtype=torch.float32, device=dev))
    Tn = torch.tensor(norm.targets(targets, kinds) * masks, dtype=torch.float32, device=dev)
    Mk = torch.tensor(masks, dtype=torch.float32, device=dev)
    P = X.shape[0]
    rng = np.random.default_rng(seed)
    history = []
    for ep in range(epochs):
        perm = torch.as_tensor(rng.permutation(P), device=dev)
        tot = torch.zeros(1, dtype=torch.float32, device=dev)
        lr_ep = lr * 0.5 * (1.0 + np.cos(np.pi * ep / epochs))  # cosine decay
        for s in range(0, P, batch):
            idx = perm[s:s + batch]
            xb, tb, mb = X[idx].contiguous(), Tn[idx].contiguous(), Mk[idx].contiguous()
            loss, grads = net.gradients(xb, tb, mb, float(mb.sum()))
            net.adam_step(grads, lr_ep)
            tot += loss * len(idx)
        history.append(float(tot) / P)
        if log:
            log(f"epoch {ep} loss {history[-1]:.4e}")
    return net, norm, history


class LearnedGuess:
    """Predicts the AO density of a water cluster; ``density`` returns None when
    the prediction fails its electron-count check (use REST's guess instead)."""

    def __init__(self, net: PairMLP, norm: Normaliser, basis: str = "def2-SVP"):
        self.net, self.norm, self.basis = net, norm, basis

    @staticmethod
    def load(path: Path = DEFAULT_WEIGHTS, device: int = 0) -> "LearnedGuess":
        st = dict(np.load(path))
        net = PairMLP(seed=0, device=device)
        net.load_state(st)
        norm = Normaliser(st["f_mean"], st["f_std"], st["t_mean"], st["t_std"])
        return LearnedGuess(net, norm, str(st["basis"]))

    def save(self, path: Path):
        st = self.net.state()
        st.update(f_mean=self.norm.f_mean, f_std=self.norm.f_std, t_mean=self.norm.t_mean, t_std=self.norm.t_std,
                  basis=np.array(self.basis))
        Path(path).parent.mkdir(parents=True, exist_ok=True)
        np.savez_compressed(path, **st)

    def _forward(self, ps: PairSet):
        import torch

        x = self.net.to_bf16(torch.tensor(self.norm.feats(ps.feats), dtype=torch.float32, device=self.net.dev))
        return self.net.forward(x)

    def predict_blocks(self, ps: PairSet) -> np.ndarray:
        y = self._forward(ps).cpu().numpy().astype(np.float64)
        return self.norm.blocks(y, ps.kind)

    def assemble_device(self, mol, sh, ps: PairSet, y):
        """The AO density from the network output y (device, standardised)
        with the library's assembly kernel; a device tensor (n x n, FP64)."""
        import torch

        dev = self.net.dev
        if not hasattr(self, "_tstats"):
            self._tstats = (torch.tensor(self.norm.t_mean, dtype=torch.float32, device=dev),
                            torch.tensor(self.norm.t_std, dtype=torch.float32, device=dev))
        up, first, typ, nfun, water, rot = (torch.as_tensor(a, device=dev) for a in assembly_inputs(mol, sh, ps))
        rot = rot.to(torch.float64)
        n = sh.nfun
        D = torch.empty(n, n, dtype=torch.float64, device=dev)
        tm, ts = self._tstats
        _ck(lib().rijk_guess_assemble(_p(y), _p(tm), _p(ts), _p(up), up.shape[0], _p(first), _p(typ), _p(nfun),
                                      _p(water), _p(rot), n, _p(D), self.net.stream), "guess_assemble")
        return D

    def write_rest_init_guess(self, mol, path, ovlp: np.ndarray | None = None) -> bool:
        """Hands the predicted density to REST's own guess path: writes the
        ``init_guess`` HDF5 file REST reads with ``external_init_guess = true``
        and ``guessfile_type = "hdf5"`` (src/initial_guess/mod.rs:17-26, :71-83),
        in REST's AO order.  Returns False (and writes nothing) when the
        prediction fails its electron-count check, so that REST keeps its own
        guess."""
        from .chkfile import write_init_guess

        d = self.density(mol, ovlp=ovlp)
        if d is None:
            return False
        # REST's closed-shell density is the total density (occupation 2), as here
        write_init_guess(path, [d], shells=mol.shells(self.basis))
        return True

    def density(self, mol, ovlp: np.ndarray | None = None, tol: float = 0.05, on_device: bool = False):
        """Predicted AO density (host array, or device tensor with on_device),
        or None when its electron count tr(D S) is off by more than ``tol``."""
        D = self.densities([mol], None if ovlp is None else [ovlp], tol)[0]
        return D if D is None or on_device else D.cpu().numpy()

    def densities(self, mols, ovlps: list | None = None, tol: float = 0.05) -> list:
        """density() for a molecule set, on the device: pair rows built by the
        geometry kernels, one network pass over the pairs of every molecule,
        one assembly launch per molecule, and one host read of all electron
        counts.  Returns device tensors (n x n, FP64), None where the
        electron-count check fails."""
        import torch

        dev = self.net.dev
        if not mols:
            return []
        if not hasattr(self, "_tstats"):
            self._tstats = (torch.tensor(self.norm.t_mean, dtype=torch.float32, device=dev),
                            torch.tensor(self.norm.t_std, dtype=torch.float32, device=dev))
        g = device_pairs(mols, self.basis, self.norm, dev)
        y = self.net.forward(self.net.to_bf16(g.feats))
        tm, ts = self._tstats
        out = []
        for i in range(len(mols)):
            p0, p1 = int(g.pair_off[i]), int(g.pair_off[i + 1])
            u0, u1 = int(g.up_off[i]), int(g.up_off[i + 1])
            a0, a1 = int(g.atom_off[i]), int(g.atom_off[i + 1])
            n = int(g.nbas[i])
            D = torch.empty(n, n, dtype=torch.float64, device=dev)
            _ck(lib().rijk_guess_assemble(_p(y[p0:p1]), _p(tm), _p(ts), _p(g.up[u0:u1]), u1 - u0,
                                          _p(g.first[a0:a1]), _p(g.typ[a0:a1]), _p(g.nfun[a0:a1]),
                                          _p(g.water[a0:a1]), _p(g.rot[a0 // 3:a1 // 3]), n, _p(D), self.net.stream),
                "guess_assemble")
            out.append(D)
        if ovlps is None:
            return out
        ne = torch.stack([(D * (S if torch.is_tensor(S) else torch.as_tensor(np.asarray(S), device=dev))).sum()
                          for D, S in zip(out, ovlps)]).cpu().numpy()
        for i, mol in enumerate(mols):
            if not np.isfinite(ne[i]) or abs(ne[i] - mol.nelec) > tol * mol.nelec:
                out[i] = None
            else:
                out[i] *= mol.nelec / ne[i]
        return out
