"""GPU-resident, batched RI-HF SCF over a set of molecules (closed shell).

Every molecule keeps its fitted tensor in its own device context (its own CUDA
stream), and the SCF iterations of the whole set advance together:

  J / K        per molecule through the device entry points (rijk_vj_upper_dev,
               rijk_vk_upper_occ_dev or the split-precision tcgen05 form), the
               molecules' launches overlapping on their streams;
  Fock, DIIS   on the device for the padded batch: F = h + J + K, the error
               vectors F D S - S D F of REST's DIIS (src/scf_io/mod.rs:3094-3136),
               the B-matrix solve of diis_solver (:3138-3188) per molecule;
  diagonalise  the generalised eigenproblem F C = S C e of diagonalize_hamiltonian
               (:1843-1873) as one batched symmetric eigensolve of X^T F X
               (X = S^-1/2 per molecule, padding rows pushed to the top of the
               spectrum) on the device;
  density      D = 2 C_occ C_occ^T on the device.

All of it is FP64.  Molecules converge independently (REST's three criteria,
:1875-1951) and stop being updated once converged.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from .basis import Molecule, int1e, int2c2e, int3c2e
from .rijk import RIJK
from .scf import metric_inv_sqrt


@dataclass
class BatchResult:
    energies: list
    converged: list
    iterations: list
    setup_s: float
    scf_s: float
    timings: dict = field(default_factory=dict)


class BatchedRHF:
    def __init__(self, mols: list, basis: str, auxbas: str, device: int = 0, metric: str = "inv_sqrt",
                 precision: str = "fp64"):
        import torch

        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.precision = precision
        t0 = time.perf_counter()
        self.mols = mols
        self.ctx, self.n, self.nocc, self.enuc = [], [], [], []
        hs, ss = [], []
        for mol in mols:
            bas, aux = mol.shells(basis), mol.shells(auxbas)
            n = bas.nfun
            s = int1e(mol, bas, "ovlp")
            h = int1e(mol, bas, "kinetic") + int1e(mol, bas, "nuclear")
            v2 = int2c2e(aux)
            i3 = int3c2e(bas, aux)
            ctx = RIJK(device)
            if metric == "inv_sqrt":
                ctx.fit_rimatr(metric_inv_sqrt(v2), i3, n)
            else:
                ctx.build_rimatr_cholesky(v2, i3, n)
            self.ctx.append(ctx)
            self.n.append(n)
            if mol.spin != 1 or mol.nelec % 2:
                raise ValueError("BatchedRHF handles closed-shell molecules")
            self.nocc.append(mol.nelec // 2)
            self.enuc.append(mol.nuclear_repulsion())
            hs.append(h)
            ss.append(s)
        self.B = len(mols)
        self.nmax = max(self.n)
        f64 = torch.float64
        B, nm = self.B, self.nmax
        self.S = torch.zeros(B, nm, nm, dtype=f64, device=self.dev)
        self.H = torch.zeros(B, nm, nm, dtype=f64, device=self.dev)
        self.X = torch.zeros(B, nm, nm, dtype=f64, device=self.dev)
        for i, (h, s) in enumerate(zip(hs, ss)):
            n = self.n[i]
            self.S[i, :n, :n] = torch.as_tensor(s, device=self.dev)
            self.H[i, :n, :n] = torch.as_tensor(h, device=self.dev)
            w, u = torch.linalg.eigh(self.S[i, :n, :n])
            self.X[i, :n, :n] = (u * w.rsqrt()) @ u.T
        # padded rows of X^T F X get a large diagonal so their eigenvalues come last
        self.pad_shift = torch.zeros(B, nm, nm, dtype=f64, device=self.dev)
        for i in range(B):
            idx = torch.arange(self.n[i], nm, device=self.dev)
            self.pad_shift[i, idx, idx] = 1.0e6
        # packed-upper <-> full index maps per size
        self._tri = {}
        self.setup_s = time.perf_counter() - t0

    def _tri_idx(self, n):
        if n not in self._tri:
            il = self.torch.tril_indices(n, n, device=self.dev)  # REST order: (i <= j), j-major
            self._tri[n] = (il[1], il[0])
        return self._tri[n]

    def _upper_to_full(self, u, n):
        i, j = self._tri_idx(n)
        m = self.torch.zeros(n, n, dtype=self.torch.float64, device=self.dev)
        m[i, j] = u
        m[j, i] = u
        return m

    def _jk(self, C, active):
        """J + K (full, padded batch) for the active molecules from their orbitals."""
        torch = self.torch
        B, nm = self.B, self.nmax
        out = torch.zeros(B, nm, nm, dtype=torch.float64, device=self.dev)
        cur = torch.cuda.current_stream()
        ev = torch.cuda.Event()
        ev.record(cur)
        parts = []
        for i in range(B):
            if not active[i]:
                continue
            ctx, n, o = self.ctx[i], self.n[i], self.nocc[i]
            st = torch.cuda.ExternalStream(ctx.stream)
            st.wait_event(ev)
            with torch.cuda.stream(st):
                c = C[i, :n, :o]
                d = 2.0 * (c @ c.T)
                c_cm = c.T.contiguous()  # column-major n x o
                occ = torch.full((o,), 2.0, dtype=torch.float64, device=self.dev)
                npair = n * (n + 1) // 2
                vj = torch.empty(npair, dtype=torch.float64, device=self.dev)
                vk = torch.empty(npair, dtype=torch.float64, device=self.dev)
                ctx.vj_upper_dev(d.contiguous().data_ptr(), 1, 1.0, 1, vj.data_ptr(), ctx.stream)
                if self.precision == "split":
                    ctx.vk_upper_occ_split_dev(c_cm.data_ptr(), o, [o - 1], occ.data_ptr(), 1, -0.5, vk.data_ptr(),
                                               ctx.stream)
                else:
                    ctx.vk_upper_occ_dev(c_cm.data_ptr(), o, [o - 1], occ.data_ptr(), 1, -0.5, vk.data_ptr(),
                                         ctx.stream)
                out[i, :n, :n] = self._upper_to_full(vj + vk, n)
                done = torch.cuda.Event()
                done.record(st)
                parts.append((done, d, c_cm, occ, vj, vk))
        for done, *_ in parts:
            cur.wait_event(done)
        return out

    def run(self, max_cycle: int = 100, acc_etot: float = 1e-8, acc_rho: float = 1e-5, acc_eev: float = 1e-5,
            num_max_diis: int = 8) -> BatchResult:
        torch = self.torch
        t0 = time.perf_counter()
        B, nm = self.B, self.nmax
        enuc = torch.tensor(self.enuc, dtype=torch.float64, device=self.dev)
        ns = torch.tensor(self.n, dtype=torch.float64, device=self.dev)
        nocc_mask = torch.zeros(B, nm, dtype=torch.float64, device=self.dev)
        for i in range(B):
            nocc_mask[i, :self.nocc[i]] = 1.0

        def diag(F):
            fp = self.X.transpose(1, 2) @ F @ self.X + self.pad_shift
            e, cp = torch.linalg.eigh(fp)
            return e, self.X @ cp

        def density(C):
            co = C * nocc_mask[:, None, :]
            return 2.0 * co @ co.transpose(1, 2)

        active = [True] * B
        e, C = diag(self.H)  # hcore guess
        D = density(C)
        F = self.H + self._jk(C, active)
        energy = enuc + 0.5 * ((D * (self.H + F)).sum(dim=(1, 2)))
        e_prev, D_prev, E_prev = e, D, energy
        errs, targets = [[] for _ in range(B)], [[] for _ in range(B)]
        iters = [0] * B
        conv = [False] * B
        for it in range(1, max_cycle + 1):
            # DIIS extrapolation of F per molecule (error F D S - S D F)
            err = F @ D @ self.S
            err = err - err.transpose(1, 2)
            Fx = F.clone()
            for i in range(B):
                if not active[i]:
                    continue
                if len(errs[i]) == num_max_diis:
                    errs[i].pop(0)
                    targets[i].pop(0)
                errs[i].append(err[i].reshape(-1))
                targets[i].append(F[i])
                E = torch.stack(errs[i])
                bm = (E @ E.T).cpu().numpy()
                try:
                    binv = np.linalg.inv(bm)
                    coef = binv.sum(axis=1) / binv.sum()
                    Fx[i] = sum(float(c) * t for c, t in zip(coef, targets[i]))
                except np.linalg.LinAlgError:
                    errs[i], targets[i] = [], []
            e, C = diag(Fx)
            Dn = density(C)
            Fn = self.H + self._jk(C, active)
            En = enuc + 0.5 * ((Dn * (self.H + Fn)).sum(dim=(1, 2)))
            de = (En - E_prev).abs()
            ddm = ((Dn - D).pow(2).sum(dim=(1, 2))).sqrt() / ns
            nmask = torch.arange(nm, device=self.dev)[None, :] < ns[:, None]
            deev = (((e - e_prev) * nmask).pow(2).sum(dim=1)).sqrt()
            de_h, ddm_h, deev_h = de.cpu().numpy(), ddm.cpu().numpy(), deev.cpu().numpy()
            for i in range(B):
                if active[i]:
                    iters[i] = it
                    if de_h[i] <= acc_etot and ddm_h[i] <= acc_rho and deev_h[i] <= acc_eev:
                        conv[i] = True
                        active[i] = False
            upd = torch.tensor([1.0 if (a or conv[i] and iters[i] == it) else 0.0 for i, a in enumerate(active)],
                               dtype=torch.float64, device=self.dev)[:, None, None]
            F = upd * Fn + (1 - upd) * F
            D = upd * Dn + (1 - upd) * D
            E_prev = torch.where(upd[:, 0, 0] > 0, En, E_prev)
            e_prev = torch.where(upd[:, :, 0] > 0, e, e_prev)
            if not any(active):
                break
        torch.cuda.synchronize()
        scf_s = time.perf_counter() - t0
        return BatchResult([float(x) for x in E_prev.cpu()], conv, iters, self.setup_s, scf_s)

    def close(self):
        for c in self.ctx:
            c.close()


def water_cluster(k: int, seed: int) -> Molecule:
    """(H2O)_k: O atoms by seeded rejection sampling in a cube of side 3.1 k^(1/3) A
    with min O-O 2.7 A; each water at the gas-phase geometry (0.9572 A, 104.52 deg)
    with a uniformly random orientation."""
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
