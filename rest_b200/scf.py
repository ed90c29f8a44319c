"""RI Hartree-Fock SCF driver around the B200 J/K build.

Restates REST's SCF loop (``scf``, src/scf_io/mod.rs:3190-3268) with the J/K
build, the metric fit and the density on the GPU through the C ABI:

  build      integrals (rest_b200.basis), overlap check (:232-244), RI metric
             (V^-1/2 as ``lapack_power(-0.5, 1e-8)``, molecule_io/mod.rs:1582, or
             the device Cholesky), fit of B on the device, initial guess
  loop       prepare_next_input (direct / linear / DIIS mixing, :2947-3091)
             -> diagonalize_hamiltonian (generalised eigenproblem, :1843-1873)
             -> generate_density_matrix (:441-478)
             -> check_scf_convergence (:1875-1951) -> update (:2910-2925)
  Fock       generate_hf_hamiltonian_ri_v (:1339-1381): F_s = h + J_a + J_b + K_s,
             J/K variant chosen as generate_vj_with_ri_v_sync / generate_vk_with_ri_v
             (:2008-2039), K scaled by -0.5 (RHF) or -1 (UHF)
  energy     E = E_nuc + 1/2 sum D (h + F) from packed storage (:1744-1802)

The generalised eigenproblem runs on the host with LAPACK, as in REST.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg as sla

from .basis import DEVICE_MAX_L_AO, DEVICE_MAX_L_AUX, Molecule, int1e, int1e_nuclear_dev, int2c2e, int2c2e_dev, int3c2e
from .rijk import RIJK

AUXBAS_THRESHOLD = 1.0e-8  # src/constants/mod.rs:81


def _upper(m: np.ndarray) -> np.ndarray:
    jj, ii = np.tril_indices(m.shape[0])
    return np.ascontiguousarray(m[ii, jj])


def _full(u: np.ndarray, n: int) -> np.ndarray:
    jj, ii = np.tril_indices(n)
    m = np.zeros((n, n))
    m[ii, jj] = u
    m[jj, ii] = u
    return m


def energy_contraction(a_upper, b_upper, n) -> float:
    """SCF::par_energy_contraction (src/scf_io/mod.rs:1787-1802)."""
    dg = np.arange(n)
    dg = dg * (dg + 1) // 2 + dg
    return (2.0 * float(np.dot(a_upper, b_upper)) - float(np.dot(a_upper[dg], b_upper[dg]))) * 0.5


def metric_inv_sqrt(v: np.ndarray, threshold: float = AUXBAS_THRESHOLD) -> np.ndarray:
    """V^-1/2 keeping eigenvalues >= threshold (lapack_power(-0.5, thr))."""
    lam, u = np.linalg.eigh(v)
    keep = lam >= threshold
    return np.asfortranarray((u[:, keep] * lam[keep] ** -0.5) @ u[:, keep].T)


def metric_inv_sqrt_dev(v) -> np.ndarray:
    """metric_inv_sqrt of a device matrix (torch, FP64): the eigendecomposition and
    the product run on the device; the factor comes back as a host array."""
    import torch

    lam, u = torch.linalg.eigh(v)
    keep = lam >= AUXBAS_THRESHOLD
    uk = u[:, keep]
    return np.asfortranarray(((uk * lam[keep].rsqrt()) @ uk.T).cpu().numpy())


@dataclass
class ScfOptions:
    """The [ctrl] keys of REST's input that steer this path (src/ctrl_io/mod.rs)."""
    use_ri_symm: bool = True
    use_dm_only: bool = False
    mixer: str = "diis"  # direct | linear | diis
    num_max_diis: int = 8
    start_diis_cycle: int = 1
    mix_param: float = 0.6
    max_scf_cycle: int = 100
    scf_acc_rho: float = 1.0e-5
    scf_acc_eev: float = 1.0e-5
    scf_acc_etot: float = 1.0e-8
    initial_guess: str = "hcore"
    metric: str = "inv_sqrt"  # inv_sqrt (REST's live path) | cholesky
    # where (P|Q) and (mu nu|P) are computed: "device" (CUDA integral engine,
    # AO l <= 2 and auxiliary l <= 4), "host" (OpenMP engine) or "auto" (device
    # when the shells are within its limits)
    integrals: str = "auto"
    start_check_oscillation: int = 20
    print_level: int = 0
    # precision of the exchange build: "fp64" (plain) or "mixed": incremental
    # split-precision (3 x BF16 on tcgen05) builds K_k = K_{k-1} + K(D_k - D_{k-1})
    # until |dE| <= mixed_switch_etot and dDM <= mixed_switch_rho, then full FP64
    # builds to convergence (the converged energy is an FP64 energy).
    precision: str = "fp64"
    # (measured on C40H82: the split error shrinks with |dD|, so hand-over at
    # |dE| <= 1e-7 with a rebuild every 16 split steps needs 6 FP64 builds instead
    # of 9 and reaches the same energy)
    mixed_switch_etot: float = 1.0e-7
    mixed_switch_rho: float = 1.0e-5
    mixed_rebuild_every: int = 16  # full FP64 rebuild of K every this many split steps


@dataclass
class ScfResult:
    energy: float
    converged: bool
    iterations: int
    eigenvalues: list
    eigenvectors: list
    density: list
    nuc_energy: float
    num_basis: int
    num_auxbas: int
    timings: dict = field(default_factory=dict)
    history: list = field(default_factory=list)


class SCF:
    def __init__(self, mol: Molecule, basis: str, auxbas: str, opts: ScfOptions | None = None,
                 ctx: RIJK | None = None, device: int = 0):
        self.mol, self.opts = mol, opts or ScfOptions()
        self.ctx = ctx or RIJK(device)
        self.basis_name, self.auxbas_name = basis, auxbas
        t0 = time.perf_counter()
        self.bas, self.aux = mol.shells(basis), mol.shells(auxbas)
        self.n, self.naux = self.bas.nfun, self.aux.nfun
        self.nuc_energy = mol.nuclear_repulsion()
        self.ovlp = int1e(mol, self.bas, "ovlp")
        if self.opts.metric not in ("inv_sqrt", "cholesky"):
            raise ValueError(f"unknown metric {self.opts.metric!r}")
        self.integrals_on = self._integral_engine()
        if self.integrals_on == "device":  # nuclear attraction through the device three-centre engine
            nuc = int1e_nuclear_dev(mol, self.bas).cpu().numpy()
        else:
            nuc = int1e(mol, self.bas, "nuclear")
        self.h_core = int1e(mol, self.bas, "kinetic") + nuc
        lam = np.linalg.eigvalsh(self.ovlp)
        if lam[0] <= 1e-10:
            raise ValueError(f"overlap matrix is singular (lowest eigenvalue {lam[0]:.3e})")
        self.ovlp_lowest_eig = float(lam[0])
        t1 = time.perf_counter()
        if self.integrals_on == "device":
            # integrals, metric and fit on the device; V^-1/2 needs V on the host
            factor = None
            if self.opts.metric == "inv_sqrt":
                factor = metric_inv_sqrt_dev(int2c2e_dev(self.aux))
            t2 = time.perf_counter()
            self.ctx.build_rimatr_from_shells(self.bas, self.aux, factor)
        else:
            v2 = int2c2e(self.aux)
            i3 = int3c2e(self.bas, self.aux)
            t2 = time.perf_counter()
            if self.opts.metric == "inv_sqrt":
                self.ctx.fit_rimatr(metric_inv_sqrt(v2), i3, self.n)
            else:
                self.ctx.build_rimatr_cholesky(v2, i3, self.n)
        t3 = time.perf_counter()
        self.timings = {"one_electron_s": t1 - t0, "ri_integrals_s": t2 - t1, "fit_s": t3 - t2}
        # occupations (generate_occupation_integer, :364-440)
        nelec = mol.nelec
        nunp = mol.spin - 1
        self.spin_channel = 1 if nunp == 0 else 2
        if self.spin_channel == 1:
            self.nelec_spin = [nelec / 2.0]
            self.occ_num = 2.0
        else:
            self.nelec_spin = [(nelec + nunp) / 2.0, (nelec - nunp) / 2.0]
            self.occ_num = 1.0
        self.k_scale = -0.5 if self.spin_channel == 1 else -1.0
        self.h_upper = _upper(self.h_core)
        # mixed-precision state: reference exchange matrix and the density terms it belongs to
        self._kref = None
        self._kref_terms = None
        self._fp64_now = self.opts.precision != "mixed"
        self._split_steps = 0
        self.split_builds = 0
        self.fp64_builds = 0

    def _integral_engine(self) -> str:
        mode = self.opts.integrals
        if mode not in ("auto", "device", "host"):
            raise ValueError(f"unknown integrals engine {mode!r}")
        if mode == "auto":
            # a context without the device builder (a CPU stand-in) takes host integrals
            fits = int(self.bas.l.max()) <= DEVICE_MAX_L_AO and int(self.aux.l.max()) <= DEVICE_MAX_L_AUX
            return "device" if fits and hasattr(self.ctx, "build_rimatr_from_shells") else "host"
        return mode

    # -- pieces of the loop ---------------------------------------------------
    def occupation(self):
        occ, homo = [], []
        for s in range(self.spin_channel):
            o = np.zeros(self.n)
            left, i = self.nelec_spin[s], 0
            while left > 0.0 and i < self.n:
                o[i] = min(left * self.occ_num, self.occ_num)
                i += 1
                left -= 1.0
            occ.append(o)
            homo.append(max(i - 1, 0))
        return occ, homo

    def diagonalize(self, fock_upper):
        vals, vecs = [], []
        for s in range(self.spin_channel):
            w, c = sla.eigh(_full(fock_upper[s], self.n), self.ovlp)
            vals.append(w)
            vecs.append(np.asfortranarray(c))
        return vals, vecs

    def density(self, eigv, occ, homo):
        return self.ctx.density_matrix(eigv, homo, occ, self.spin_channel)

    # -- mixed precision: exchange of a density difference ---------------------
    def terms_of(self, eigv, occ, homo):
        """Factor terms of a density: D_s = sum coef Y Y^T with Y = C[:, :nw] sqrt(occ)."""
        return [[(1.0, np.asarray(eigv[s])[:, :homo[s] + 1] * np.sqrt(np.asarray(occ[s])[:homo[s] + 1]))]
                for s in range(self.spin_channel)]

    @staticmethod
    def mix_terms(t0, t1, alpha):
        return [[(c * (1.0 - alpha), y) for c, y in a] + [(c * alpha, y) for c, y in b] for a, b in zip(t0, t1)]

    def delta_factor(self, terms_new, terms_ref):
        """dD = sum_new - sum_ref as V S V^T with V = Q U |lam|^1/2 (thin QR of the
        stacked factors, eigendecomposition of the small core), positive columns first."""
        cols, sg = [], []
        for sign, terms in ((1.0, terms_new), (-1.0, terms_ref)):
            for c, y in terms:
                cc = sign * c
                if cc == 0.0 or y.shape[1] == 0:
                    continue
                cols.append(np.sqrt(abs(cc)) * y)
                sg.append(np.full(y.shape[1], np.sign(cc)))
        if not cols:
            return np.zeros((self.n, 0)), 0
        w = np.hstack(cols)
        s = np.concatenate(sg)
        q, r = np.linalg.qr(w)
        lam, u = np.linalg.eigh((r * s) @ r.T)
        big = np.max(np.abs(lam)) if lam.size else 0.0
        keep = np.abs(lam) > 1e-14 * max(big, 1e-300)
        lam, u = lam[keep], u[:, keep]
        order = np.argsort(-lam)  # positive eigenvalues first
        lam, u = lam[order], u[:, order]
        v = (q @ u) * np.sqrt(np.abs(lam))
        return v, int(np.sum(lam > 0))

    def k_split_delta(self, terms_new, terms_ref):
        """K_s(D_new - D_ref) for each spin by the split-precision tcgen05 build."""
        import torch

        out = []
        n, ld = self.n, self.n + (self.n & 1)
        st = self.ctx.stream
        with torch.cuda.stream(torch.cuda.ExternalStream(st)):
            for s in range(self.spin_channel):
                v, npos = self.delta_factor(terms_new[s], terms_ref[s])
                dk = torch.zeros(self.n * (self.n + 1) // 2, dtype=torch.float64, device="cuda")
                if v.shape[1] > 0:
                    buf = np.zeros((v.shape[1], ld))
                    buf[:, :n] = v.T
                    dv = torch.tensor(buf, dtype=torch.float64, device="cuda")
                    self.ctx.vk_upper_lowrank_split_dev(dv.data_ptr(), ld, v.shape[1], npos, self.k_scale, False,
                                                        dk.data_ptr(), st)
                self.ctx.synchronize(st)
                out.append(dk.cpu().numpy())
        return out

    def hamiltonian(self, dm, eigv=None, occ=None, homo=None, terms=None):
        """generate_hf_hamiltonian_ri_v + the energy of generate_hf_hamiltonian."""
        sc = self.spin_channel
        o = self.opts
        incremental = (o.precision == "mixed" and terms is not None and getattr(self, "_kref", None) is not None
                       and not self._fp64_now and self._split_steps < o.mixed_rebuild_every)
        if o.use_ri_symm:
            vj = self.ctx.vj_upper_with_rimatr_v(dm, sc, 1.0)
        else:
            vj = self.ctx.vj_upper_with_ri_v(dm, sc, 1.0)
        if incremental:
            dk = self.k_split_delta(terms, self._kref_terms)
            vk = [self._kref[s] + dk[s] for s in range(sc)] + [np.zeros(1)] * (2 - sc)
            self._split_steps += 1
            self.split_builds += 1
        else:
            if o.use_ri_symm:
                vk = self.ctx.vk_upper_with_rimatr_use_dm_only(dm, sc, self.k_scale)
            elif o.use_dm_only or eigv is None:
                vk = self.ctx.vk_upper_with_ri_v_use_dm_only(dm, sc, self.k_scale)
            else:
                vk = self.ctx.vk_upper_with_ri_v(eigv, homo, occ, sc, self.k_scale)
            self._split_steps = 0
            self.fp64_builds += 1
        if o.precision == "mixed" and terms is not None:
            self._kref = [vk[s].copy() for s in range(sc)]
            self._kref_terms = terms
        fock = []
        for s in range(sc):
            f = self.h_upper.copy()
            for j in vj:
                if j.size == f.size:
                    f = f + j
            fock.append(f + vk[s])
        e = self.nuc_energy
        if sc == 1:
            e += energy_contraction(_upper(dm[0]), self.h_upper + fock[0], self.n)
        else:
            da, db = _upper(dm[0]), _upper(dm[1])
            e += energy_contraction(da + db, self.h_upper, self.n)
            e += energy_contraction(da, fock[0], self.n) + energy_contraction(db, fock[1], self.n)
        return fock, e

    def initial_density(self):
        """REST's initial_guess (src/initial_guess/mod.rs:15-80): 'hcore'
        diagonalises the core Hamiltonian; 'sad' builds the Fock matrix of the
        superposed atomic densities (dm-only exchange), diagonalises it and
        takes the density of its orbitals (:46-58)."""
        if self.opts.initial_guess == "sad":
            from .sad import sad_density

            make = getattr(self.ctx, "spawn", None)
            dm0 = sad_density(self.mol, self.basis_name, self.auxbas_name, make)
            fock, _ = self.hamiltonian(dm0)
            vals, vecs = self.diagonalize(fock)
        elif self.opts.initial_guess == "hcore":
            vals, vecs = self.diagonalize([self.h_upper] * self.spin_channel)
        else:
            raise ValueError("bundled initial guesses: 'hcore', 'sad'")
        occ, homo = self.occupation()
        return self.density(vecs, occ, homo), vecs, occ, homo

    # -- the loop -------------------------------------------------------------
    def run(self) -> ScfResult:
        o = self.opts
        t0 = time.perf_counter()
        n, sc = self.n, self.spin_channel
        dm, eigv, occ, homo = self.initial_density()
        terms0 = self.terms_of(eigv, occ, homo)
        fock, energy = self.hamiltonian(dm, eigv, occ, homo, terms=terms0)
        vals, eigv = self.diagonalize(fock)
        occ, homo = self.occupation()
        dm_new = self.density(eigv, occ, homo)
        # ScfTraceRecord: density_matrix = [previous, current input]
        rec_dm = [dm, dm_new]
        rec_terms = [terms0, self.terms_of(eigv, occ, homo)]
        fp64_streak = 0
        rec_energy, rec_vals = energy, vals
        num_iter = 1
        start_diis = o.start_diis_cycle
        err_vecs, targets, energies, history = [], [], [], []
        prev_fock = None
        converged = False
        s_full = self.ovlp
        while True:
            # prepare_next_input
            dm_in = rec_dm[1]
            fp64_before = self.fp64_builds
            if o.mixer == "direct":
                fock, energy = self.hamiltonian(dm_in, eigv, occ, homo, terms=rec_terms[1])
            elif o.mixer == "linear" or (o.mixer == "diis" and num_iter < start_diis):
                dm_in = [rec_dm[0][s] + o.mix_param * (rec_dm[1][s] - rec_dm[0][s]) for s in range(sc)]
                fock, energy = self.hamiltonian(dm_in, eigv, occ, homo,
                                                terms=self.mix_terms(rec_terms[0], rec_terms[1], o.mix_param))
            else:
                fock, energy = self.hamiltonian(dm_in, eigv, occ, homo, terms=rec_terms[1])
                energies.append(energy)
                osc = len(energies) >= 2 and len(energies) > o.start_check_oscillation and energies[-1] > energies[-2]
                if len(targets) == o.num_max_diis:
                    targets.pop(0)
                    err_vecs.pop(0)
                ev, tg = [], []
                for s in range(sc):
                    f = _full(fock[s], n)
                    d = rec_dm[1][s]
                    ev.append((f @ d @ s_full - s_full @ d @ f).ravel())
                    tg.append(f)
                err_vecs.append(np.concatenate(ev))
                targets.append(tg)
                bmat = np.array([[np.dot(a, b) for b in err_vecs] for a in err_vecs])
                try:
                    binv = np.linalg.inv(bmat)
                    if not np.all(np.isfinite(binv)):
                        raise np.linalg.LinAlgError
                    coeff = binv.sum(axis=1) / binv.sum()
                    new = []
                    for s in range(sc):
                        hm = sum(c * t[s] for c, t in zip(coeff, targets))
                        hu = _upper(hm)
                        if osc and prev_fock is not None:
                            hu = (1.0 - o.mix_param) * prev_fock[s] + o.mix_param * hu
                        new.append(hu)
                    fock = new
                    prev_fock = fock
                except np.linalg.LinAlgError:
                    dm_in = [rec_dm[0][s] + o.mix_param * (rec_dm[1][s] - rec_dm[0][s]) for s in range(sc)]
                    fock, energy = self.hamiltonian(dm_in, eigv, occ, homo,
                                                    terms=self.mix_terms(rec_terms[0], rec_terms[1], o.mix_param))
                    start_diis = num_iter + 8
                    err_vecs, targets = [], []
            fp64_streak = fp64_streak + 1 if self.fp64_builds > fp64_before else 0
            vals, eigv = self.diagonalize(fock)
            occ, homo = self.occupation()
            dm_new = self.density(eigv, occ, homo)
            terms_new = self.terms_of(eigv, occ, homo)
            # check_scf_convergence against the record
            de = energy - rec_energy
            eev = float(np.sqrt(sum(np.sum((vals[s] - rec_vals[s]) ** 2) for s in range(sc))))
            ddm = [float(np.sqrt(np.sum((dm_new[s] - rec_dm[1][s]) ** 2)) / n) for s in range(sc)]
            history.append({"iter": num_iter, "energy": energy, "d_energy": de, "d_dm": ddm, "d_eev": eev})
            if o.print_level > 0:
                print(f"Energy: {energy:18.10f} Ha after {num_iter:4d} iterations; "
                      f"dDM {max(ddm):.3e} deev {eev:.3e} dE {de:.3e}")
            conv = num_iter >= 2 and abs(de) <= o.scf_acc_etot and max(ddm) <= o.scf_acc_rho and eev <= o.scf_acc_eev
            if o.precision == "mixed":
                # converged only on consecutive full FP64 builds; leave the split
                # builds once the SCF is loosely converged
                conv = conv and fp64_streak >= 2
                if not self._fp64_now and abs(de) <= o.mixed_switch_etot and max(ddm) <= o.mixed_switch_rho:
                    self._fp64_now = True
            # update
            rec_dm = [rec_dm[1], dm_new]
            rec_terms = [rec_terms[1], terms_new]
            rec_energy, rec_vals = energy, vals
            num_iter += 1
            if conv:
                converged = True
                break
            if num_iter > o.max_scf_cycle:
                break
        self.timings["scf_s"] = time.perf_counter() - t0
        self.timings["fp64_k_builds"] = self.fp64_builds
        self.timings["split_k_builds"] = self.split_builds
        return ScfResult(energy, converged, num_iter - 1, vals, eigv, rec_dm[1], self.nuc_energy, n, self.naux,
                         dict(self.timings), history)


def rhf_energy(mol: Molecule, basis: str, auxbas: str, **kw) -> ScfResult:
    ctx = kw.pop("ctx", None)
    return SCF(mol, basis, auxbas, ScfOptions(**kw), ctx=ctx).run()
