"""GPU-resident, batched RI-HF SCF over a set of molecules (closed shell).

Every molecule keeps its fitted tensor in its own device context (its own CUDA
stream), and the SCF iterations of the whole set advance together:

  integrals    (P|Q), (mu nu|P), metric and fit on the device per molecule
               (rijk_build_rimatr_from_shells) when the shells fit the device
               engine, else the host engine; the molecules' setups run on a pool
               of host threads (``setup_workers``), each with its own stream, so
               that one molecule's host-side plan and one-electron integrals
               overlap the others' device work;
  J / K        FP64 builds of a group of molecules (``grouped``) by the
               library's grouped build (rijk_group_jk_occ_dev: six launches for
               all of them, captured once in a CUDA graph and replayed every
               iteration with the converged molecules switched off); otherwise
               per molecule through the device entry points
               (rijk_vjk_upper_occ_dev, which takes J from the K half-transform,
               or the split-precision tcgen05 forms), the molecules' launches
               overlapping on their streams;
  Fock, DIIS   on the device for the padded batch: F = h + J + K, the error
               vectors F D S - S D F of REST's DIIS (src/scf_io/mod.rs:3094-3136)
               kept as a batched history, the B matrices of diis_solver
               (:3138-3188) formed in one batched product and solved for all
               molecules by one launch (rijk_diis_coefficients_dev);
  diagonalise  the generalised eigenproblem F C = S C e of diagonalize_hamiltonian
               (:1843-1873) in the standard form X^T F X with X = L^-T from the
               Cholesky factor S = L L^T (the reduction of REST's LAPACK dspgvx),
               padding rows pushed to the top of the spectrum; each molecule's
               eigenbasis from the previous iteration is refined by matrix
               products (eigsolve.refine), and molecules where that does not
               pass take the library's batched eigensolver
               (rijk_eigh_batched_dev; cuSOLVER for a matrix it does not
               converge or one beyond its size limit);
  density      D = 2 C_occ C_occ^T on the device.

Precision of the exchange build:
  fp64   every K in FP64 (DMMA);
  mixed  for molecules with at least ``split_min_basis`` (512) basis functions,
         incremental split-precision J and K: K_k = K_{k-1} + K_split(D_k - D_{k-1})
         and J_k = J_{k-1} + J(D_k - D_{k-1}), J's aux-row scalars taken from the
         split half-transform of the difference (one FP64 pass over the tensor
         instead of two), with
         the density difference in its exact low-rank form V S V^T (batched thin
         QR of [Y_k, Y_{k-1}] and an eigendecomposition of the small core, so the
         split error scales with |dD|), a full FP64 rebuild every
         ``rebuild_every`` split steps, FP64 builds once the molecule is loosely
         converged, and convergence only on consecutive FP64 builds, so every
         reported energy is an FP64 energy; smaller molecules take FP64 builds;
  split  every K in split precision (no FP64 finish; for loose criteria only).
Everything else is FP64.  Molecules converge independently (REST's three
criteria, :1875-1951) and stop being updated once converged.
"""
from __future__ import annotations

import os
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from .basis import DEVICE_MAX_L_AO, DEVICE_MAX_L_AUX, int1e, int1e_nuclear_dev, int2c2e, int2c2e_dev, int3c2e
from .geometry import alkane, water_cluster  # noqa: F401  (re-exported)
from .rijk import RIJK, RIJKGroup, group_tiles
from .eigsolve import diis_coefficients, eigh_batched, refine
from .scf import metric_inv_sqrt, metric_inv_sqrt_dev


def host_blas_limit(threads: int | None):
    """Cap the host BLAS thread pools (numpy's and scipy's OpenBLAS) for the
    duration of a ``with`` block, restoring them afterwards; None leaves them.
    The batched driver's host BLAS work is a handful of tiny products per
    iteration, done between device calls from several host threads: with the
    pools at their default of one thread per core, their spinning workers
    compete with those threads (measured on a 16-core host, 64 water clusters
    from the learned guess: 10.8 molecules/s with the defaults, 22.2 with one
    BLAS thread)."""
    import contextlib

    if threads is None:
        return contextlib.nullcontext()
    try:
        from threadpoolctl import threadpool_limits
    except ImportError:  # without threadpoolctl the pools keep their sizes
        return contextlib.nullcontext()
    return threadpool_limits(limits=int(threads), user_api="blas")


@dataclass
class BatchResult:
    energies: list
    converged: list
    iterations: list
    setup_s: float
    scf_s: float
    timings: dict = field(default_factory=dict)
    densities: list = field(default_factory=list)  # converged AO densities (host), when asked for


class BatchedRHF:
    def __init__(self, mols: list, basis: str, auxbas: str, device: int = 0, metric: str = "inv_sqrt",
                 precision: str = "fp64", integrals: str = "auto", rebuild_every: int = 16,
                 switch_etot: float = 1e-7, switch_rho: float = 1e-5, eig_workers: int = 8,
                 graphs: bool = False, split_min_basis: int = 512, refine_eigs: bool = True,
                 setup_workers: int = 8, host_blas_threads: int | None = 1, contexts: list | None = None,
                 grouped: bool = True, group_graphs: bool = True, native_eigh: bool | None = None):
        import torch

        if precision not in ("fp64", "mixed", "split"):
            raise ValueError(f"unknown precision {precision!r}")
        if metric not in ("inv_sqrt", "cholesky"):
            raise ValueError(f"unknown metric {metric!r}")
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.precision = precision
        self.rebuild_every, self.switch_etot, self.switch_rho = rebuild_every, switch_etot, switch_rho
        # split-precision K pays only where K dominates: measured on B200, below
        # about 500 basis functions the operand preparation and the low-rank
        # factorisation of dD cost more than the split build saves
        self.split_min_basis = split_min_basis
        self.eig_workers, self._pool = eig_workers, None
        # eigenbases of the previous iteration refined by matrix products
        # (eigsolve.refine); a fresh eigensolve only where that does not pass
        self.refine_eigs = refine_eigs
        # fresh eigensolves on the library's batched solver (cuSOLVER as its
        # fallback); RIJK_NATIVE_EIGH=0 selects cuSOLVER alone
        if native_eigh is None:
            native_eigh = os.environ.get("RIJK_NATIVE_EIGH", "1") != "0"
        self.native_eigh = native_eigh
        self._vbasis, self._have_basis = None, []
        self._eig_counts = {"refined": 0, "eigh": 0}
        # CUDA graphs of the per-molecule FP64 J/K (orbital form), captured after
        # the first build with every context's buffers pinned
        self.graphs = graphs and precision == "fp64"
        self._graph = None
        self.host_blas_threads = host_blas_threads
        # contexts lent by the caller (one per molecule, at least as many as
        # molecules): their tensors are replaced here, and close() leaves them open
        if contexts is not None and len(contexts) < len(mols):
            raise ValueError("fewer contexts than molecules")
        self._borrowed = contexts is not None
        with host_blas_limit(host_blas_threads):
            self._setup(mols, basis, auxbas, device, metric, integrals, setup_workers, contexts)
        # Grouped FP64 build: every molecule's J + K in one set of launches
        # (rijk_group_*), tile shapes from the autotuner on the largest molecule,
        # captured once in a CUDA graph and replayed every iteration.  It serves
        # every build when no molecule takes split-precision steps.
        self._group, self._ggraph = None, None
        self.group_graphs = group_graphs
        all_fp64 = precision == "fp64" or (precision == "mixed" and max(self.n) < split_min_basis)
        if grouped and all_fp64:
            t0 = time.perf_counter()
            big = max(range(self.B), key=lambda i: self.n[i])
            tiles = group_tiles(self.ctx[big], self.nocc[big], sample_rows=256)
            self._group = RIJKGroup(self.ctx, self.nocc, *tiles)
            self.setup_parts["group"] = time.perf_counter() - t0
            self.setup_s += self.setup_parts["group"]

    def _setup(self, mols, basis, auxbas, device, metric, integrals, setup_workers, contexts):
        import torch

        t0 = time.perf_counter()
        self.mols = mols
        for mol in mols:
            if mol.spin != 1 or mol.nelec % 2:
                raise ValueError("BatchedRHF handles closed-shell molecules")
        # torch loads its device linear-algebra backend on first use, and that
        # first use must not happen on several threads at once (setup and
        # eigensolve threads): load it here
        with torch.cuda.device(self.dev):
            torch.linalg.eigh(torch.eye(2, dtype=torch.float64, device=self.dev))
        tls = threading.local()

        def one(i, mol):
            """One molecule's context and integrals (host one-electron parts,
            device nuclear attraction, device three-centre integrals, metric and
            fit), on this thread's own stream; returns when its device work is done."""
            part = {"host_one_electron": 0.0, "contexts": 0.0, "device": 0.0}
            if not hasattr(tls, "stream"):
                tls.stream = torch.cuda.Stream(device=self.dev)
            with torch.cuda.device(self.dev), torch.cuda.stream(tls.stream):
                bas, aux = mol.shells(basis), mol.shells(auxbas)
                n = bas.nfun
                ta = time.perf_counter()
                s = int1e(mol, bas, "ovlp")
                on_device = integrals == "device" or (
                    integrals == "auto" and int(bas.l.max()) <= DEVICE_MAX_L_AO and int(aux.l.max()) <= DEVICE_MAX_L_AUX)
                tk = int1e(mol, bas, "kinetic") if on_device else None
                tb = time.perf_counter()
                ctx = contexts[i] if contexts is not None else RIJK(device)
                tc = time.perf_counter()
                part["host_one_electron"] += tb - ta
                part["contexts"] += tc - tb
                try:
                    if on_device:  # kinetic on the host, nuclear attraction and the tensor on the device
                        h = torch.as_tensor(tk, device=self.dev) + int1e_nuclear_dev(mol, bas)
                        factor = metric_inv_sqrt_dev(int2c2e_dev(aux)) if metric == "inv_sqrt" else None
                        ctx.build_rimatr_from_shells(bas, aux, factor)
                    else:
                        h = int1e(mol, bas, "kinetic") + int1e(mol, bas, "nuclear")
                        v2, i3 = int2c2e(aux), int3c2e(bas, aux)
                        if metric == "inv_sqrt":
                            ctx.fit_rimatr(metric_inv_sqrt(v2), i3, n)
                        else:
                            ctx.build_rimatr_cholesky(v2, i3, n)
                    tls.stream.synchronize()
                except BaseException:
                    if contexts is None:
                        ctx.close()
                    raise
                part["device"] += time.perf_counter() - tc
            return ctx, n, h, s, part

        nw = max(1, min(setup_workers, len(mols)))
        if nw == 1:
            outs = [one(i, m) for i, m in enumerate(mols)]
        else:
            from concurrent.futures import ThreadPoolExecutor

            with ThreadPoolExecutor(nw) as pool:
                futs = [pool.submit(one, i, m) for i, m in enumerate(mols)]
                outs, err = [], None
                for f in futs:
                    try:
                        outs.append(f.result())
                    except BaseException as e:  # noqa: BLE001  (closed below, then re-raised)
                        err = err or e
            if err is not None:
                if contexts is None:
                    for o in outs:
                        o[0].close()
                raise err
        # host time per phase, summed over the setup threads
        parts = {"host_one_electron": 0.0, "contexts": 0.0, "device": 0.0}
        for o in outs:
            for k, v in o[4].items():
                parts[k] += v
        parts["molecules_wall"] = time.perf_counter() - t0
        self.ctx = [o[0] for o in outs]
        self.n = [o[1] for o in outs]
        self.nocc = [m.nelec // 2 for m in mols]
        self.enuc = [m.nuclear_repulsion() for m in mols]
        hs = [o[2] for o in outs]
        ss = [o[3] for o in outs]
        self.B = len(mols)
        self.nmax = max(self.n)
        self.omax = max(self.nocc)
        f64 = torch.float64
        B, nm = self.B, self.nmax
        self.S = torch.zeros(B, nm, nm, dtype=f64, device=self.dev)
        self.H = torch.zeros(B, nm, nm, dtype=f64, device=self.dev)
        for i, (h, s) in enumerate(zip(hs, ss)):
            n = self.n[i]
            self.S[i, :n, :n] = torch.as_tensor(s, device=self.dev)
            self.H[i, :n, :n] = torch.as_tensor(h, device=self.dev)
        pad_eye = torch.zeros(B, nm, nm, dtype=f64, device=self.dev)
        for i in range(B):
            idx = torch.arange(self.n[i], nm, device=self.dev)
            pad_eye[i, idx, idx] = 1.0
        # X = L^-T from S = L L^T (identity on the padding): the reduction to a
        # standard eigenproblem that REST's packed generalised solver performs
        # (LAPACK dspgvx, src/scf_io/mod.rs:1851), batched; an S that is not
        # numerically positive definite takes X = S^-1/2 instead
        td = time.perf_counter()
        L, info = torch.linalg.cholesky_ex(self.S + pad_eye)
        if bool((info != 0).any()):
            w, u = torch.linalg.eigh(self.S + pad_eye)
            self.X = (u * w.rsqrt()[:, None, :]) @ u.transpose(1, 2) - pad_eye
        else:
            eye = torch.eye(nm, dtype=f64, device=self.dev).expand(B, nm, nm)
            self.X = torch.linalg.solve_triangular(L, eye, upper=False).transpose(1, 2) - pad_eye
        # padded rows of X^T F X get a large diagonal so their eigenvalues come last
        self.pad_shift = 1.0e6 * pad_eye
        self._pad_eye = pad_eye
        self._have_basis = [False] * B
        self._tri = {}
        for n in sorted(set(self.n)):
            self._tri_idx(n)
        parts["orthogonaliser_submit"] = time.perf_counter() - td
        td = time.perf_counter()
        torch.cuda.synchronize()
        parts["device_wait"] = time.perf_counter() - td
        self.setup_parts = parts
        self.setup_s = time.perf_counter() - t0

    def _eigh(self, fp, nvalid=None):
        """Batched symmetric eigensolve: the library's solver (one CTA per
        matrix, rijk_eigh_batched_dev) for batches of at least 16 matrices, with
        cuSOLVER for a matrix it reports as not converged, one beyond its size
        limit, and batches of fewer matrices (one CTA per matrix would leave most
        of the GPU idle; in the alkane runs, one molecule per batch, a 490 x 490
        eigensolve on one SM made each SCF iteration several times slower)."""
        torch = self.torch
        if nvalid is not None and fp.shape[1] <= 768 and self.native_eigh and fp.shape[0] >= 16:
            lam, V, ok = eigh_batched(fp, nvalid, pad_value=1.0e6)
            bad = torch.nonzero(~ok).flatten().tolist()
            if bad:
                bi = torch.as_tensor(bad, device=self.dev)
                lb, vb = self._eigh_cusolver(fp[bi])
                lam[bi], V[bi] = lb, vb
                self._eig_counts["cusolver"] = self._eig_counts.get("cusolver", 0) + len(bad)
            return lam, V
        return self._eigh_cusolver(fp)

    def _eigh_cusolver(self, fp):
        """Batched symmetric eigensolve through cuSOLVER, split over several
        streams from host threads: each cuSOLVER call is a chain of small kernels,
        and chains on different streams overlap on the GPU."""
        torch = self.torch
        nw = min(self.eig_workers, fp.shape[0])
        if nw <= 1:
            return torch.linalg.eigh(fp)
        if self._pool is None:
            from concurrent.futures import ThreadPoolExecutor

            self._pool = ThreadPoolExecutor(self.eig_workers)
            self._eig_streams = [torch.cuda.Stream(device=self.dev) for _ in range(self.eig_workers)]
        main = torch.cuda.current_stream()
        ready = torch.cuda.Event()
        ready.record(main)
        bounds = np.linspace(0, fp.shape[0], nw + 1).astype(int)

        def work(j):
            st = self._eig_streams[j]
            st.wait_event(ready)
            with torch.cuda.stream(st):
                part = fp[bounds[j]:bounds[j + 1]]
                e, v = torch.linalg.eigh(part)
                done = torch.cuda.Event()
                done.record(st)
            part.record_stream(st)
            e.record_stream(main)
            v.record_stream(main)
            return e, v, done

        res = list(self._pool.map(work, range(nw)))
        for _, _, done in res:
            main.wait_event(done)
        return torch.cat([e for e, _, _ in res]), torch.cat([v for _, v, _ in res])

    def _solve(self, A, rows):
        """Eigenpairs of the orthogonalised Fock matrices A (one per molecule of
        ``rows``): molecules with an eigenbasis from the previous iteration
        refine it (4 steps, 5 more while still converging); the rest, and those
        whose refinement does not pass, take a fresh eigensolve.  The bases are
        kept, with the padded block set to the identity, for the next call."""
        torch = self.torch
        nr, nm = A.shape[0], A.shape[1]
        e_r = torch.empty(nr, nm, dtype=A.dtype, device=self.dev)
        cp = torch.empty(nr, nm, nm, dtype=A.dtype, device=self.dev)
        done = [False] * nr
        loc = [k for k, i in enumerate(rows) if self._have_basis[i]] if self.refine_eigs else []
        if loc:
            li = torch.as_tensor(loc, device=self.dev)
            nv = [self.n[rows[k]] for k in loc]
            gi = torch.as_tensor([rows[k] for k in loc], device=self.dev)
            lam, V, ok, off = refine(A[li], self._vbasis[gi], nv, steps=4)
            ok_h, off_h = ok.cpu().numpy(), off.cpu().numpy()
            more = [j for j in range(len(loc)) if not ok_h[j] and off_h[j] < 1e-2]
            if more:
                mj = torch.as_tensor(more, device=self.dev)
                lam2, V2, ok2, _ = refine(A[li[mj]], V[mj], [nv[j] for j in more], steps=5)
                lam[mj], V[mj] = lam2, V2
                for j, o in zip(more, ok2.cpu().numpy()):
                    ok_h[j] = o
            e_r[li], cp[li] = lam, V
            for j, k in enumerate(loc):
                done[k] = bool(ok_h[j])
        todo = [k for k in range(nr) if not done[k]]
        if todo:
            ti = torch.as_tensor(todo, device=self.dev)
            e_t, v_t = self._eigh(A[ti], [self.n[rows[k]] for k in todo])
            e_r[ti], cp[ti] = e_t, v_t
        self._eig_counts["refined"] += nr - len(todo)
        self._eig_counts["eigh"] += len(todo)
        if self.refine_eigs:
            r = torch.as_tensor(rows, device=self.dev)
            if self._vbasis is None:
                self._vbasis = torch.zeros(self.B, nm, nm, dtype=A.dtype, device=self.dev)
            pe = self._pad_eye[r]
            keep = (pe.diagonal(dim1=1, dim2=2) == 0).to(A.dtype)
            self._vbasis[r] = cp * keep[:, :, None] * keep[:, None, :] + pe
            for i in rows:
                self._have_basis[i] = True
        return e_r, cp

    def _tri_idx(self, n):
        """Row and column of each packed upper-triangle element for size n.  The
        per-molecule streams of the J/K dispatch read these cached tensors without
        waiting on the stream that made them, so they are made on the calling
        stream and synchronised before first use (the constructor makes every
        size of the batch)."""
        if n not in self._tri:
            torch = self.torch
            il = torch.tril_indices(n, n, device=self.dev)  # REST order: (i <= j), j-major
            torch.cuda.current_stream(self.dev).synchronize()
            self._tri[n] = (il[1], il[0])
        return self._tri[n]

    def _upper_to_full(self, u, n):
        i, j = self._tri_idx(n)
        m = self.torch.zeros(n, n, dtype=self.torch.float64, device=self.dev)
        m[i, j] = u
        m[j, i] = u
        return m

    def _delta_factors(self, Y, idx):
        """For molecules idx: dD = Y Y^T - Yref Yref^T as V S V^T, V = Q U |lam|^1/2
        with positive columns first (batched thin QR + eigensolve of the 2o x 2o core)."""
        torch = self.torch
        om = self.omax
        Yn = Y[idx]
        Yr = torch.stack([self._yref[i] for i in idx])
        W = torch.cat([Yn, Yr], dim=2)
        Q, R = torch.linalg.qr(W)
        sgn = torch.cat([torch.ones(om, dtype=W.dtype, device=self.dev), -torch.ones(om, dtype=W.dtype, device=self.dev)])
        M = (R * sgn[None, None, :]) @ R.transpose(1, 2)
        lam, U = torch.linalg.eigh(M)
        lam_h = lam.cpu().numpy()
        out = {}
        for b, i in enumerate(idx):
            lb = lam_h[b]
            big = np.max(np.abs(lb)) if lb.size else 0.0
            keep = np.nonzero(np.abs(lb) > 1e-14 * max(big, 1e-300))[0]
            keep = keep[np.argsort(-lb[keep])]
            if keep.size == 0:
                out[i] = (None, 0)
                continue
            kt = torch.as_tensor(keep, device=self.dev)
            sq = torch.as_tensor(np.sqrt(np.abs(lb[keep])), dtype=W.dtype, device=self.dev)
            V = (Q[b] @ U[b][:, kt]) * sq[None, :]
            out[i] = (V[:self.n[i]], int(np.sum(lb[keep] > 0)))
        return out

    def _capture(self):
        """One CUDA graph per molecule: D = 2 C C^T, J and K through the device
        entry points on the molecule's capture stream, unpacked into a static
        padded output.  Inputs are read from a static orbital buffer."""
        torch = self.torch
        B, nm, om = self.B, self.nmax, self.omax
        self._gC = torch.zeros(B, nm, om, dtype=torch.float64, device=self.dev)
        self._gout = torch.zeros(B, nm, nm, dtype=torch.float64, device=self.dev)
        self._gocc = torch.full((om,), 2.0, dtype=torch.float64, device=self.dev)
        self._graph = []
        for i in range(B):
            ctx, n, o = self.ctx[i], self.n[i], self.nocc[i]
            self._tri_idx(n)
            st = torch.cuda.Stream(device=self.dev)
            npair = n * (n + 1) // 2

            def body():
                c_cm = self._gC[i, :n, :o].T.contiguous()
                vj = torch.empty(npair, dtype=torch.float64, device=self.dev)
                vk = torch.empty(npair, dtype=torch.float64, device=self.dev)
                # J of D = 2 C C^T and K from one build (J's scalars from the K half-transform)
                ctx.vjk_upper_occ_dev(c_cm.data_ptr(), o, [o - 1], self._gocc.data_ptr(), 1, 1.0, -0.5,
                                      vj.data_ptr(), vk.data_ptr(), st.cuda_stream)
                self._gout[i, :n, :n] = self._upper_to_full(vj + vk, n)

            st.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(st):
                body()  # warm-up on the capture stream (library scratch already sized)
            st.synchronize()
            ctx.pin_buffers(True)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=st):
                body()
            self._graph.append((g, st))
        torch.cuda.synchronize()

    def _jk_replay(self, C, active):
        torch = self.torch
        self._gC.copy_(C[:, :, :self.omax] * self._occ_mask[:, None, :self.omax])
        cur = torch.cuda.current_stream()
        ev = torch.cuda.Event()
        ev.record(cur)
        for i in range(self.B):
            if not active[i]:
                continue
            g, st = self._graph[i]
            st.wait_event(ev)
            with torch.cuda.stream(st):
                g.replay()
            done = torch.cuda.Event()
            done.record(st)
            cur.wait_event(done)
            self._nfp64[i] += 1
            self._streak[i] += 1
        return self._gout.clone()

    def _jk_group(self, C, active):
        """J + K of the active molecules by the grouped build (graph replay)."""
        torch = self.torch
        B, nm = self.B, self.nmax
        act = torch.tensor([1 if a else 0 for a in active], dtype=torch.int32, device=self.dev)
        args = (nm * nm, nm, 1, -0.5)
        if not self.group_graphs:
            out = torch.zeros(B, nm, nm, dtype=torch.float64, device=self.dev)
            self._group.jk_occ_dev(C.contiguous().data_ptr(), *args, act.data_ptr(), out.data_ptr(), nm * nm, nm,
                                   torch.cuda.current_stream().cuda_stream)
        else:
            if self._ggraph is None:
                self._gsC = torch.zeros(B, nm, nm, dtype=torch.float64, device=self.dev)
                self._gsA = torch.zeros(B, dtype=torch.int32, device=self.dev)
                self._gsO = torch.zeros(B, nm, nm, dtype=torch.float64, device=self.dev)
                st = torch.cuda.Stream(device=self.dev)

                def call():
                    self._group.jk_occ_dev(self._gsC.data_ptr(), *args, self._gsA.data_ptr(), self._gsO.data_ptr(),
                                           nm * nm, nm, st.cuda_stream)

                st.wait_stream(torch.cuda.current_stream())
                with torch.cuda.stream(st):
                    call()  # warm-up outside the capture (function attributes, module load)
                st.synchronize()
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=st):
                    call()
                self._ggraph = g
            self._gsC.copy_(C)
            self._gsA.copy_(act)
            self._ggraph.replay()
            out = self._gsO.clone()
        for i in range(B):
            if active[i]:
                self._nfp64[i] += 1
                self._streak[i] += 1
        return out

    def _jk(self, C, active):
        """J + K (full, padded batch) for the active molecules from their orbitals."""
        if self._group is not None:
            return self._jk_group(C, active)
        if self._graph is not None:
            return self._jk_replay(C, active)
        torch = self.torch
        B, nm, om = self.B, self.nmax, self.omax
        out = torch.zeros(B, nm, nm, dtype=torch.float64, device=self.dev)
        Y = np.sqrt(2.0) * C[:, :, :om] * self._occ_mask[:, None, :om]  # D = Y Y^T
        incr = [self.precision == "mixed" and active[i] and self._kref[i] is not None and not self._fp64_now[i]
                and self._split_steps[i] < self.rebuild_every for i in range(B)]
        factors = self._delta_factors(Y, [i for i in range(B) if incr[i]]) if any(incr) else {}
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
                npair = n * (n + 1) // 2
                vj = torch.empty(npair, dtype=torch.float64, device=self.dev)
                keep = [vj]
                if self.precision == "split":
                    d = (2.0 * (c @ c.T)).contiguous()
                    ctx.vj_upper_dev(d.data_ptr(), 1, 1.0, 1, vj.data_ptr(), ctx.stream)
                    keep.append(d)
                if incr[i]:
                    # J and K of the density difference in split precision, added to the
                    # previous build's: J_k = J_ref + J(dD), K_k = K_ref + K(dD)
                    vk = self._kref[i].clone()
                    vj.copy_(self._jref[i])
                    V, npos = factors[i]
                    if V is not None:
                        ld = n + (n & 1)
                        buf = torch.zeros(V.shape[1], ld, dtype=torch.float64, device=self.dev)
                        buf[:, :n] = V.T
                        vjd = torch.empty(npair, dtype=torch.float64, device=self.dev)
                        ctx.vjk_upper_lowrank_split_dev(buf.data_ptr(), ld, V.shape[1], npos, 1.0, -0.5, True,
                                                        vjd.data_ptr(), vk.data_ptr(), ctx.stream)
                        vj.add_(vjd)
                        keep += [buf, vjd]
                    self._split_steps[i] += 1
                    self._nsplit[i] += 1
                    self._streak[i] = 0
                else:
                    c_cm = c.T.contiguous()  # column-major n x o
                    occ = torch.full((o,), 2.0, dtype=torch.float64, device=self.dev)
                    vk = torch.empty(npair, dtype=torch.float64, device=self.dev)
                    if self.precision == "split":
                        ctx.vk_upper_occ_split_dev(c_cm.data_ptr(), o, [o - 1], occ.data_ptr(), 1, -0.5,
                                                   vk.data_ptr(), ctx.stream)
                        self._nsplit[i] += 1
                    else:
                        # J of D = 2 C C^T and K from one build
                        ctx.vjk_upper_occ_dev(c_cm.data_ptr(), o, [o - 1], occ.data_ptr(), 1, 1.0, -0.5,
                                              vj.data_ptr(), vk.data_ptr(), ctx.stream)
                        self._nfp64[i] += 1
                        self._streak[i] += 1
                    self._split_steps[i] = 0
                    keep += [c_cm, occ]
                if self.precision == "mixed":
                    self._kref[i] = vk
                    self._jref[i] = vj
                    self._yref[i] = Y[i].clone()
                out[i, :n, :n] = self._upper_to_full(vj + vk, n)
                done = torch.cuda.Event()
                done.record(st)
                parts.append((done, keep, vk))
        for done, *_ in parts:
            cur.wait_event(done)
        return out

    def _jk_dm(self, D, which):
        """J + K from densities (REST's dm-only exchange, a4/a5) for molecules in
        ``which``: the first build from a supplied initial density."""
        torch = self.torch
        B, nm = self.B, self.nmax
        out = torch.zeros(B, nm, nm, dtype=torch.float64, device=self.dev)
        cur = torch.cuda.current_stream()
        ev = torch.cuda.Event()
        ev.record(cur)
        parts = []
        for i in range(B):
            if not which[i]:
                continue
            ctx, n = self.ctx[i], self.n[i]
            st = torch.cuda.ExternalStream(ctx.stream)
            st.wait_event(ev)
            with torch.cuda.stream(st):
                d = D[i, :n, :n].contiguous()
                npair = n * (n + 1) // 2
                vj = torch.empty(npair, dtype=torch.float64, device=self.dev)
                vk = torch.empty(npair, dtype=torch.float64, device=self.dev)
                ctx.vj_upper_dev(d.data_ptr(), 1, 1.0, 1, vj.data_ptr(), ctx.stream)
                ctx.vk_upper_dm_dev(d.data_ptr(), 1, -0.5, vk.data_ptr(), ctx.stream)
                self._nfp64[i] += 1
                self._streak[i] += 1
                out[i, :n, :n] = self._upper_to_full(vj + vk, n)
                done = torch.cuda.Event()
                done.record(st)
                parts.append((done, d, vj, vk))
        for done, *_ in parts:
            cur.wait_event(done)
        return out

    def run(self, max_cycle: int = 100, acc_etot: float = 1e-8, acc_rho: float = 1e-5, acc_eev: float = 1e-5,
            num_max_diis: int = 8, initial_densities: list | None = None,
            return_densities: bool = False, guess=None) -> BatchResult:
        """Converge every molecule.  ``initial_densities``: per molecule an AO
        density (n x n) to start from, or None for REST's hcore guess.
        ``guess``: a model with ``density(mol, ovlp=S, on_device=True)`` (the
        learned guess) that supplies the densities instead, checked against the
        overlap matrices already on the device; a molecule whose prediction
        fails the check starts from hcore."""
        if guess is not None:
            t0 = time.perf_counter()
            initial_densities = guess.densities(self.mols, [self.S[i, :self.n[i], :self.n[i]]
                                                            for i in range(len(self.mols))])
            self.setup_parts["guess"] = self.setup_parts.get("guess", 0.0) + time.perf_counter() - t0
            self.setup_parts["guess_fallbacks"] = self.setup_parts.get("guess_fallbacks", 0) + sum(
                d is None for d in initial_densities)
        with host_blas_limit(self.host_blas_threads):
            return self._run(max_cycle, acc_etot, acc_rho, acc_eev, num_max_diis, initial_densities,
                             return_densities)

    def _run(self, max_cycle, acc_etot, acc_rho, acc_eev, num_max_diis, initial_densities, return_densities):
        torch = self.torch
        t0 = time.perf_counter()
        B, nm = self.B, self.nmax
        f64 = torch.float64
        enuc = torch.tensor(self.enuc, dtype=f64, device=self.dev)
        ns = torch.tensor(self.n, dtype=f64, device=self.dev)
        self._occ_mask = torch.zeros(B, nm, dtype=f64, device=self.dev)
        for i in range(B):
            self._occ_mask[i, :self.nocc[i]] = 1.0
        self._kref, self._jref, self._yref = [None] * B, [None] * B, [None] * B
        self._split_steps, self._nsplit, self._nfp64, self._streak = [0] * B, [0] * B, [0] * B, [0] * B
        self._fp64_now = [self.precision != "mixed" or self.n[i] < self.split_min_basis for i in range(B)]
        nmask = torch.arange(nm, device=self.dev)[None, :] < ns[:, None]

        def diag(F, rows=None):
            """Eigenpairs of the molecules in ``rows`` (all when None); the other
            rows of the result are zero and are not used."""
            rows = list(range(B)) if rows is None else rows
            r = torch.as_tensor(rows, device=self.dev)
            Xr = self.X[r]
            e_r, cp = self._solve(Xr.transpose(1, 2) @ F[r] @ Xr + self.pad_shift[r], rows)
            e = torch.zeros(B, nm, dtype=f64, device=self.dev)
            C = torch.zeros(B, nm, nm, dtype=f64, device=self.dev)
            e[r] = e_r
            C[r] = Xr @ cp
            return e, C

        def density(C):
            co = C * self._occ_mask[:, None, :]
            return 2.0 * co @ co.transpose(1, 2)

        active = [True] * B
        given = [d is not None for d in (initial_densities or [None] * B)]
        hc = [i for i in range(B) if not given[i]]  # hcore guess where no density is given
        if hc:
            e, C = diag(self.H, hc)
        else:
            e = torch.zeros(B, nm, dtype=f64, device=self.dev)
            C = torch.zeros(B, nm, nm, dtype=f64, device=self.dev)
        D = density(C)
        for i in range(B):
            if given[i]:
                n = self.n[i]
                D[i] = 0.0
                d0 = initial_densities[i]
                D[i, :n, :n] = d0 if torch.is_tensor(d0) else torch.as_tensor(np.asarray(d0), dtype=f64,
                                                                               device=self.dev)
        F = self.H + self._jk(C, [not g for g in given])
        if any(given):
            F = F + self._jk_dm(D, given)
        if self.graphs and self._graph is None:
            self._capture()
        E_prev = enuc + 0.5 * ((D * (self.H + F)).sum(dim=(1, 2)))
        e_prev = e
        # DIIS history as a ring buffer per molecule
        m = num_max_diis
        err_hist = torch.zeros(B, m, nm * nm, dtype=f64, device=self.dev)
        f_hist = torch.zeros(B, m, nm, nm, dtype=f64, device=self.dev)
        count = [0] * B
        iters = [0] * B
        conv = [False] * B
        # host time between the loop's own synchronisation points
        tp = {"diis": 0.0, "eigensolve": 0.0, "fock_build": 0.0}
        for it in range(1, max_cycle + 1):
            ta = time.perf_counter()
            err = F @ D @ self.S
            err = err - err.transpose(1, 2)
            act = torch.tensor(active, device=self.dev)
            # the active molecules' rows as an index built on the host: no
            # device-to-host synchronisation (a boolean mask would need one)
            live = [i for i in range(B) if active[i]]
            rows = torch.tensor(live, device=self.dev)
            slot = torch.tensor([count[i] % m for i in live], device=self.dev)
            err_hist[rows, slot] = err.index_select(0, rows).reshape(len(live), -1)
            f_hist[rows, slot] = F.index_select(0, rows)
            for i in range(B):
                if active[i]:
                    count[i] += 1
            bm = err_hist @ err_hist.transpose(1, 2)
            # REST's diis_solver per molecule, on the device (rijk_diis_coefficients_dev)
            coef, failed = diis_coefficients(bm, [count[i] if active[i] else 0 for i in range(B)])
            for i in torch.nonzero(failed).flatten().tolist():
                # singular B: restart the history from the newest Fock matrix (coefficients (1, 0, ...))
                last = (count[i] - 1) % m
                err_hist[i, 0] = err_hist[i, last].clone()
                f_hist[i, 0] = f_hist[i, last].clone()
                err_hist[i, 1:] = 0.0
                f_hist[i, 1:] = 0.0
                count[i] = 1
            tb = time.perf_counter()
            Fx = torch.einsum("bm,bmij->bij", coef, f_hist)
            Fx = torch.where(act[:, None, None], Fx, F)
            e, C = diag(Fx, [i for i in range(B) if active[i]])
            tc = time.perf_counter()
            Dn = density(C)
            Fn = self.H + self._jk(C, active)
            En = enuc + 0.5 * ((Dn * (self.H + Fn)).sum(dim=(1, 2)))
            de = (En - E_prev).abs()
            ddm = ((Dn - D).pow(2).sum(dim=(1, 2))).sqrt() / ns
            deev = (((e - e_prev) * nmask).pow(2).sum(dim=1)).sqrt()
            de_h, ddm_h, deev_h = de.cpu().numpy(), ddm.cpu().numpy(), deev.cpu().numpy()
            td = time.perf_counter()
            tp["diis"] += tb - ta
            tp["eigensolve"] += tc - tb
            tp["fock_build"] += td - tc
            newly = []
            for i in range(B):
                if not active[i]:
                    continue
                iters[i] = it
                ok = de_h[i] <= acc_etot and ddm_h[i] <= acc_rho and deev_h[i] <= acc_eev
                if self.precision == "mixed":
                    ok = ok and self._streak[i] >= 2
                    if not self._fp64_now[i] and de_h[i] <= self.switch_etot and ddm_h[i] <= self.switch_rho:
                        self._fp64_now[i] = True
                if ok:
                    conv[i] = True
                    newly.append(i)
            upd = torch.tensor([1.0 if active[i] else 0.0 for i in range(B)], dtype=f64, device=self.dev)
            F = torch.where(upd[:, None, None] > 0, Fn, F)
            D = torch.where(upd[:, None, None] > 0, Dn, D)
            E_prev = torch.where(upd > 0, En, E_prev)
            e_prev = torch.where(upd[:, None] > 0, e, e_prev)
            for i in newly:
                active[i] = False
            if not any(active):
                break
        # a converged density must hold the electrons and be idempotent
        # (D S D = 2 D); a molecule that fails either is reported as not converged
        ne = (D * self.S).sum(dim=(1, 2))
        idem = (D @ self.S @ D - 2.0 * D).abs().amax(dim=(1, 2))
        ne_h, idem_h = ne.cpu().numpy(), idem.cpu().numpy()
        checks = []
        for i in range(B):
            ok = bool(abs(ne_h[i] - 2 * self.nocc[i]) < 1e-6 * max(1, 2 * self.nocc[i]) and idem_h[i] < 1e-6)
            checks.append(ok)
            conv[i] = bool(conv[i] and ok)
        torch.cuda.synchronize()
        scf_s = time.perf_counter() - t0
        timings = {"fp64_k_builds": list(self._nfp64), "split_k_builds": list(self._nsplit),
                   "density_checks": checks, "eigensolves": dict(self._eig_counts),
                   "setup_parts": dict(self.setup_parts), "scf_parts": tp}
        dens = [D[i, :self.n[i], :self.n[i]].cpu().numpy() for i in range(B)] if return_densities else []
        return BatchResult([float(x) for x in E_prev.cpu()], conv, iters, self.setup_s, scf_s, timings, dens)

    def close(self):
        self._graph = None  # graphs go before the contexts whose memory they use
        self._ggraph = None
        if self._group is not None:
            self.torch.cuda.synchronize(self.dev)
            self._group.close()
            self._group = None
        if self._pool is not None:
            self._pool.shutdown()
            self._pool = None
        for c in self.ctx:
            if self._borrowed:
                c.pin_buffers(False)  # pinned for graph replay; the lender may load other tensors
            else:
                c.close()
        self.ctx = []


def device_bytes(n: int, naux: int, nocc: int, precision: str = "fp64") -> int:
    """Device memory one molecule's context holds during the SCF: the tile-packed
    tensor, the half-transform scratch (capped at the context's 4 GiB budget),
    and for split precision the BF16 hi/lo copies of the full B_P."""
    nt = -(-n // 32)
    naux_pad = -(-naux // 32) * 32
    tensor = naux_pad * (nt * (nt + 1) // 2 * 1024) * 8
    ldx = -(-n // 128) * 128
    scratch = min(4 << 30, naux * ldx * (-(-nocc // 128) * 128) * 8)
    split = naux_pad * ldx * ldx * 4 if precision in ("mixed", "split") else 0
    group = naux * nocc * ldx * 8  # the grouped build's half-transform scratch
    return tensor + scratch + split + group + 8 * n * n * 8


def pool_reuse(held: list, needs: list, budget: float) -> int:
    """How many pooled contexts a group keeps.  ``held``: the memory each pooled
    context holds (the largest molecule it served), ``needs``: the group's
    molecules, largest first, paired with the pool in order.  Reusing keeps
    min(len(held), len(needs)) contexts, each then holding the larger of the
    two, plus fresh contexts for the rest; if that exceeds ``budget`` the pool
    is dropped (0) and the group starts afresh."""
    keep = min(len(held), len(needs))
    cost = sum(max(held[j], needs[j]) for j in range(keep)) + sum(needs[keep:])
    return keep if cost <= budget else 0


def run_molecule_set(mols: list, basis: str, auxbas: str, group_size: int = 64, device: int = 0,
                     metric: str = "cholesky", memory_fraction: float = 0.5, **kw) -> BatchResult:
    """Converge a molecule set in groups of at most ``group_size`` molecules of
    similar size (sorted by basis size so that padding stays small) whose
    estimated device memory stays within ``memory_fraction`` of the memory free
    at the start; the groups run one after another on the device, results come
    back in the input order.  The metric defaults to the device Cholesky fit (no
    host eigendecomposition)."""
    import torch

    kw["metric"] = metric
    run_kw = {k: kw.pop(k) for k in ("max_cycle", "acc_etot", "acc_rho", "acc_eev", "num_max_diis",
                                      "return_densities") if k in kw}
    guesses = kw.pop("initial_densities", None)
    model = kw.pop("guess", None)
    sizes = [m.shells(basis).nfun for m in mols]
    order = sorted(range(len(mols)), key=lambda i: sizes[i])
    torch.cuda.empty_cache()
    budget = memory_fraction * torch.cuda.mem_get_info(device)[0]
    prec = kw.get("precision", "fp64")
    need = {i: device_bytes(sizes[i], mols[i].shells(auxbas).nfun, mols[i].nelec // 2, prec) for i in order}
    groups, cur, used = [], [], 0
    for i in order:  # consecutive molecules of similar size, within the count and memory limits
        if cur and (len(cur) == group_size or used + need[i] > budget):
            groups.append(cur)
            cur, used = [], 0
        cur.append(i)
        used += need[i]
    if cur:
        groups.append(cur)
    energies, conv, iters = [None] * len(mols), [False] * len(mols), [0] * len(mols)
    nfp64, nsplit = [0] * len(mols), [0] * len(mols)
    dens = [None] * len(mols) if run_kw.get("return_densities") else []
    setup = scf = 0.0
    eig = {"refined": 0, "eigh": 0}
    parts = {}
    teardown = 0.0
    # One set of contexts serves the groups, largest molecules first: a context
    # keeps its tensor and scratch allocations when a smaller molecule replaces
    # its tensor, so a later group allocates nothing new.  What a pooled context
    # holds is the estimate for the largest molecule it served; a group reuses
    # the pool only while held plus new memory stays within the budget, else
    # the pool is closed and the group starts afresh.
    pool, held = [], []
    group_iters = 0  # batched iterations run: per group, its slowest molecule's count
    try:
        for idx in reversed(groups):
            idx = sorted(idx, key=lambda i: -need[i])
            keep = pool_reuse(held, [need[i] for i in idx], budget)
            tt = time.perf_counter()
            for c in pool[keep:]:
                c.close()
            pool, held = pool[:keep], held[:keep]
            teardown += time.perf_counter() - tt
            while len(pool) < len(idx):
                pool.append(RIJK(device))
                held.append(0)
            for j, i in enumerate(idx):
                held[j] = max(held[j], need[i])
            b = BatchedRHF([mols[i] for i in idx], basis, auxbas, device=device, contexts=pool[:len(idx)], **kw)
            try:
                r = b.run(initial_densities=None if guesses is None else [guesses[i] for i in idx], guess=model,
                          **run_kw)
            finally:
                # the next group reuses torch's cached blocks: releasing them here
                # would only make it allocate them again
                tt = time.perf_counter()
                b.close()
                teardown += time.perf_counter() - tt
            setup += r.setup_s
            scf += r.scf_s
            group_iters += max(r.iterations) if r.iterations else 0
            for k in eig:
                eig[k] += r.timings["eigensolves"][k]
            for k, v in list(r.timings["setup_parts"].items()) + list(r.timings["scf_parts"].items()):
                parts[k] = parts.get(k, 0.0) + v
            for j, i in enumerate(idx):
                energies[i], conv[i], iters[i] = r.energies[j], r.converged[j], r.iterations[j]
                nfp64[i], nsplit[i] = r.timings["fp64_k_builds"][j], r.timings["split_k_builds"][j]
                if dens:
                    dens[i] = r.densities[j]
    finally:
        tt = time.perf_counter()
        for c in pool:
            c.close()
        torch.cuda.empty_cache()
        teardown += time.perf_counter() - tt
    parts["teardown"] = teardown
    parts["groups"] = len(groups)
    parts["group_iterations"] = group_iters
    parts["free_bytes_at_start"] = float(budget / memory_fraction)
    return BatchResult(energies, conv, iters, setup, scf,
                       {"fp64_k_builds": nfp64, "split_k_builds": nsplit, "eigensolves": eig, "setup_parts": parts},
                       dens)
