"""Host-side mirror of REST's RI J/K interface over the C ABI.

``RIJK`` owns one device context holding the fitted tensor (REST's
``SCF::rimatr`` / ``SCF::ri3fn``).  Its methods carry the names, argument
meaning and return shapes of REST's free functions in ``src/scf_io/mod.rs``:
they take spin-resolved lists of column-major (Fortran-order) matrices and
return a list of two packed upper triangles (``MatrixUpper``), the second a
one-element placeholder when ``spin_channel == 1`` -- exactly as REST does.
Errors raise ``RijkError`` (REST panics).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._abi import RijkError, lib


def _f64(a, shape=None) -> np.ndarray:
    a = np.asarray(a, dtype=np.float64)
    if shape is not None and a.shape != shape:
        raise ValueError(f"expected shape {shape}, got {a.shape}")
    return a


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def _stack_spin(mats, spin_channel: int, shape) -> np.ndarray:
    """Spin-resolved list -> one contiguous buffer of column-major matrices."""
    out = np.empty((spin_channel,) + tuple(reversed(shape)), dtype=np.float64)
    for s in range(spin_channel):
        m = _f64(mats[s], tuple(shape))
        out[s] = m.T  # row-major view of the transpose == column-major data
    return out


def _rest_list(parts):
    """REST returns Vec of length 2 with a 1-element placeholder in slot 1."""
    out = list(parts)
    while len(out) < 2:
        out.append(np.zeros(1))
    return out


TILE_CFGS = 6  # CTA shapes of the K kernels (RIJK_TILE_CFGS in include/rest_b200.h)


class RIJK:
    """A device context holding one fitted three-centre tensor."""

    def __init__(self, device: int = 0):
        L = lib()
        h = C.c_void_p()
        st = L.rijk_ctx_create(int(device), C.byref(h))
        if st != 0:
            raise RijkError(st, f"cannot open an sm_100 context on device {device}")
        self._h = h
        self.device = int(device)
        self.num_basis = 0
        self.num_auxbas = 0

    def spawn(self) -> "RIJK":
        """Another context on the same device (for a side calculation that must
        not replace this context's tensor, such as the atoms of the SAD guess)."""
        return RIJK(self.device)

    # -- plumbing ----------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            lib().rijk_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def _check(self, st: int, failed_pivot: int = 0):
        if st != 0:
            msg = lib().rijk_ctx_last_error(self._h)
            raise RijkError(st, msg.decode() if msg else "", failed_pivot)

    @property
    def npair(self) -> int:
        return self.num_basis * (self.num_basis + 1) // 2

    @property
    def stream(self) -> int:
        return lib().rijk_ctx_stream(self._h) or 0

    def tensor_bytes(self) -> int:
        b = C.c_int64()
        self._check(lib().rijk_ctx_info(self._h, None, None, C.byref(b)))
        return b.value

    PROF_CLASSES = ("j_pass1", "j_pass2", "j_other", "k_half", "k_rank", "k_dm", "k_other")

    def pin_buffers(self, pinned: bool = True):
        """Freeze the context's device memory (for CUDA graph capture of *_dev calls)."""
        self._check(lib().rijk_ctx_pin_buffers(self._h, int(bool(pinned))))

    def set_wait_budget(self, nanoseconds: int = 0):
        """Budget of every device-side wait of this context (0 = default 2 s)."""
        self._check(lib().rijk_ctx_set_wait_budget(self._h, int(nanoseconds)))

    def selftest_timeout(self):
        """Run one bounded wait that nothing completes; raises RijkError with
        status RIJK_ERR_TIMEOUT when the timeout path works."""
        self._check(lib().rijk_ctx_selftest_timeout(self._h))

    def set_tiles(self, half_transform_cfg: int, update_cfg: int):
        self._check(lib().rijk_ctx_set_tiles(self._h, int(half_transform_cfg), int(update_cfg)))

    def tiles(self):
        """(half-transform shape, update shape) currently selected."""
        h, u = C.c_int(), C.c_int()
        self._check(lib().rijk_ctx_get_tiles(self._h, C.byref(h), C.byref(u)))
        return h.value, u.value

    def shape(self):
        """(num_basis, num_auxbas) of the loaded tensor (0, 0 when none)."""
        n, naux = C.c_int64(), C.c_int64()
        self._check(lib().rijk_ctx_info(self._h, C.byref(n), C.byref(naux), None))
        return n.value, naux.value

    def autotune(self, ncols: int, sample_rows: int = 0):
        """Time every CTA shape on this tensor, keep the fastest; returns
        (half_cfg, update_cfg, {cfg: (half_ms, update_ms)})."""
        bh, br = C.c_int(), C.c_int()
        ms = (C.c_double * (2 * TILE_CFGS))()
        self._check(lib().rijk_ctx_autotune(self._h, int(ncols), int(sample_rows), C.byref(bh), C.byref(br), ms))
        return bh.value, br.value, {c: (ms[2 * c], ms[2 * c + 1]) for c in range(TILE_CFGS)}

    def profile(self, enable: bool = True):
        self._check(lib().rijk_ctx_profile(self._h, int(bool(enable))))

    def profile_read(self) -> dict:
        """{class: (milliseconds, launches)} accumulated since the last read."""
        k = len(self.PROF_CLASSES)
        ms = (C.c_double * k)()
        cnt = (C.c_int64 * k)()
        self._check(lib().rijk_ctx_profile_read(self._h, ms, cnt))
        return {name: (ms[i], cnt[i]) for i, name in enumerate(self.PROF_CLASSES)}

    @staticmethod
    def kernel_launches() -> int:
        return int(lib().rijk_kernel_launches())

    def synchronize(self, stream: int = 0):
        self._check(lib().rijk_ctx_synchronize(self._h, C.c_void_p(stream or None)))

    # -- fitted tensor -----------------------------------------------------
    def set_rimatr(self, rimatr: np.ndarray, num_basis: int):
        """rimatr: MatrixFull[npair, N] (Fortran order)."""
        npair = num_basis * (num_basis + 1) // 2
        r = np.asfortranarray(_f64(rimatr))
        if r.shape[0] != npair:
            raise ValueError("rimatr must have num_basis*(num_basis+1)/2 rows")
        self._check(lib().rijk_set_rimatr(self._h, _ptr(r), num_basis, r.shape[1]))
        self.num_basis, self.num_auxbas = num_basis, r.shape[1]

    def set_ri3fn(self, ri3fn: np.ndarray):
        """ri3fn: RIFull[n, n, N] (Fortran order)."""
        r = np.asfortranarray(_f64(ri3fn))
        n, n2, naux = r.shape
        if n != n2:
            raise ValueError("ri3fn must be n x n x N")
        self._check(lib().rijk_set_ri3fn(self._h, _ptr(r), n, naux))
        self.num_basis, self.num_auxbas = n, naux

    def tensor_ptr(self) -> tuple[int, int]:
        """(device address, row stride in doubles) of the tile-packed tensor."""
        p = C.c_void_p()
        ld = C.c_int64()
        self._check(lib().rijk_ctx_tensor(self._h, C.byref(p), C.byref(ld)))
        return int(p.value), int(ld.value)

    def tensor_alloc(self, num_basis: int, num_auxbas: int):
        self._check(lib().rijk_tensor_alloc(self._h, num_basis, num_auxbas))
        self.num_basis, self.num_auxbas = num_basis, num_auxbas

    def tensor_load_rows_dev(self, d_rows: int, p0: int, np_rows: int, layout: int = 0, stream: int = 0):
        self._check(lib().rijk_tensor_load_rows_dev(self._h, C.c_void_p(d_rows), p0, np_rows, layout,
                                                    C.c_void_p(stream or None)))

    def get_rimatr(self) -> np.ndarray:
        out = np.empty((self.npair, self.num_auxbas), order="F")
        self._check(lib().rijk_get_rimatr(self._h, _ptr(out)))
        return out

    def build_rimatr_cholesky(self, aux_v: np.ndarray, int3c: np.ndarray, num_basis: int):
        """Metric V = L L^T and B = int3c L^-T on the device."""
        v = np.asfortranarray(_f64(aux_v))
        m = np.asfortranarray(_f64(int3c))
        piv = C.c_int64(0)
        st = lib().rijk_build_rimatr_cholesky(self._h, _ptr(v), _ptr(m), num_basis, m.shape[1], C.byref(piv))
        self._check(st, piv.value)
        self.num_basis, self.num_auxbas = num_basis, m.shape[1]

    def fit_rimatr(self, metric_factor: np.ndarray, int3c: np.ndarray, num_basis: int):
        """B = int3c M for a caller-supplied factor (e.g. REST's V^-1/2)."""
        f = np.asfortranarray(_f64(metric_factor))
        m = np.asfortranarray(_f64(int3c))
        self._check(lib().rijk_fit_rimatr(self._h, _ptr(f), _ptr(m), num_basis, m.shape[1]))
        self.num_basis, self.num_auxbas = num_basis, m.shape[1]

    def build_rimatr_from_shells(self, bas, aux, metric_factor: np.ndarray | None = None):
        """Integrals, metric and fit all on the device (REST's
        prepare_rimatr_for_ri_v_rayon_v02): Cholesky fit when ``metric_factor``
        is None, else B = (mu nu|P) M with the given factor (e.g. V^-1/2).
        ``bas`` and ``aux`` are ``basis.ShellSet`` objects."""
        from .basis import _C2S_PTRS

        piv = C.c_int64(0)
        f = None if metric_factor is None else np.asfortranarray(_f64(metric_factor))
        st = lib().rijk_build_rimatr_from_shells(self._h, C.byref(bas.cstruct()), C.byref(aux.cstruct()),
                                                 _C2S_PTRS, None if f is None else _ptr(f), C.byref(piv))
        self._check(st, piv.value)
        self.num_basis, self.num_auxbas = bas.nfun, aux.nfun

    # -- J -------------------------------------------------------------------
    def _vj(self, fn, dm, spin_channel, scaling_factor, full=False):
        n = self.num_basis
        d = _stack_spin(dm, spin_channel, (n, n))
        per = n * n if full else self.npair
        out = np.empty(spin_channel * per)
        self._check(fn(self._h, _ptr(d), spin_channel, float(scaling_factor), _ptr(out)))
        if full:
            return _rest_list([out[s * per:(s + 1) * per].reshape(n, n, order="F") for s in range(spin_channel)])
        return _rest_list([out[s * per:(s + 1) * per].copy() for s in range(spin_channel)])

    def vj_upper_with_ri_v(self, dm, spin_channel: int, scaling_factor: float):
        """REST ``vj_upper_with_ri_v_sync`` (scf_io/mod.rs:2428)."""
        return self._vj(lib().rijk_vj_upper_with_ri_v, dm, spin_channel, scaling_factor)

    def vj_upper_with_rimatr_v(self, dm, spin_channel: int, scaling_factor: float):
        """REST ``vj_upper_with_rimatr_v_sync`` (scf_io/mod.rs:2490)."""
        return self._vj(lib().rijk_vj_upper_with_rimatr_v, dm, spin_channel, scaling_factor)

    def vj_full_with_ri_v(self, dm, spin_channel: int, scaling_factor: float):
        """REST ``vj_full_with_ri_v`` (scf_io/mod.rs:2564)."""
        return self._vj(lib().rijk_vj_full_with_ri_v, dm, spin_channel, scaling_factor, full=True)

    # -- K -------------------------------------------------------------------
    def vk_upper_with_ri_v(self, eigv, homo, occupation, spin_channel: int, scaling_factor: float):
        """REST ``vk_upper_with_ri_v_sync`` (scf_io/mod.rs:2758): occupied-orbital form."""
        n = self.num_basis
        num_state = np.asarray(eigv[0]).shape[1]
        c = _stack_spin(eigv, spin_channel, (n, num_state))
        occ = np.ascontiguousarray(np.stack([_f64(occupation[s])[:num_state] for s in range(spin_channel)]))
        hm = (C.c_int64 * 2)(*[int(homo[s]) if s < spin_channel else 0 for s in range(2)])
        out = np.empty(spin_channel * self.npair)
        st = lib().rijk_vk_upper_with_ri_v(
            self._h, _ptr(c), num_state, hm, _ptr(occ), spin_channel, float(scaling_factor), _ptr(out)
        )
        self._check(st)
        p = self.npair
        return _rest_list([out[s * p:(s + 1) * p].copy() for s in range(spin_channel)])

    def vjk_upper_with_ri_v(self, eigv, homo, occupation, spin_channel: int, j_scaling_factor: float,
                            k_scaling_factor: float):
        """J and K of REST ``generate_hf_hamiltonian_ri_v`` (scf_io/mod.rs:1339-1381)
        in one build: (vj, vk) with vj of dm_s = C_s diag(occ_s) C_s^T (the
        states up to homo) and vk as ``vk_upper_with_ri_v``."""
        n = self.num_basis
        num_state = np.asarray(eigv[0]).shape[1]
        c = _stack_spin(eigv, spin_channel, (n, num_state))
        occ = np.ascontiguousarray(np.stack([_f64(occupation[s])[:num_state] for s in range(spin_channel)]))
        hm = (C.c_int64 * 2)(*[int(homo[s]) if s < spin_channel else 0 for s in range(2)])
        vj = np.empty(spin_channel * self.npair)
        vk = np.empty(spin_channel * self.npair)
        self._check(lib().rijk_vjk_upper_with_ri_v(self._h, _ptr(c), num_state, hm, _ptr(occ), spin_channel,
                                                   float(j_scaling_factor), float(k_scaling_factor), _ptr(vj),
                                                   _ptr(vk)))
        p = self.npair
        return (_rest_list([vj[s * p:(s + 1) * p].copy() for s in range(spin_channel)]),
                _rest_list([vk[s * p:(s + 1) * p].copy() for s in range(spin_channel)]))

    def _vk_dm(self, fn, dm, spin_channel, scaling_factor, full=False):
        n = self.num_basis
        d = _stack_spin(dm, spin_channel, (n, n))
        per = n * n if full else self.npair
        out = np.empty(spin_channel * per)
        self._check(fn(self._h, _ptr(d), spin_channel, float(scaling_factor), _ptr(out)))
        if full:
            return _rest_list([out[s * per:(s + 1) * per].reshape(n, n, order="F") for s in range(spin_channel)])
        return _rest_list([out[s * per:(s + 1) * per].copy() for s in range(spin_channel)])

    def vk_upper_with_ri_v_use_dm_only(self, dm, spin_channel: int, scaling_factor: float):
        """REST ``vk_upper_with_ri_v_use_dm_only_sync`` (scf_io/mod.rs:2640)."""
        return self._vk_dm(lib().rijk_vk_upper_with_ri_v_use_dm_only, dm, spin_channel, scaling_factor)

    def vk_upper_with_rimatr_use_dm_only(self, dm, spin_channel: int, scaling_factor: float):
        """REST ``vk_upper_with_rimatr_use_dm_only_sync`` (scf_io/mod.rs:2703)."""
        return self._vk_dm(lib().rijk_vk_upper_with_rimatr_use_dm_only, dm, spin_channel, scaling_factor)

    def vk_full_fromdm_with_ri_v(self, dm, spin_channel: int, scaling_factor: float):
        """REST ``vk_full_fromdm_with_ri_v`` (scf_io/mod.rs:2603)."""
        return self._vk_dm(lib().rijk_vk_full_fromdm_with_ri_v, dm, spin_channel, scaling_factor, full=True)

    # -- device-resident forms (raw device pointers, e.g. torch .data_ptr()) --
    def vj_upper_dev(self, d_dm: int, spin_channel: int, scaling_factor: float, dm_mode: int, d_vj: int,
                     stream: int = 0):
        self._check(lib().rijk_vj_upper_dev(self._h, C.c_void_p(d_dm), spin_channel, float(scaling_factor),
                                            int(dm_mode), C.c_void_p(d_vj), C.c_void_p(stream or None)))

    def vk_upper_occ_dev(self, d_eigv: int, num_state: int, homo, d_occ: int, spin_channel: int,
                         scaling_factor: float, d_vk: int, stream: int = 0):
        hm = (C.c_int64 * 2)(*[int(homo[s]) if s < spin_channel else 0 for s in range(2)])
        self._check(lib().rijk_vk_upper_occ_dev(self._h, C.c_void_p(d_eigv), num_state, hm, C.c_void_p(d_occ),
                                                spin_channel, float(scaling_factor), C.c_void_p(d_vk),
                                                C.c_void_p(stream or None)))

    def vjk_upper_occ_dev(self, d_eigv: int, num_state: int, homo, d_occ: int, spin_channel: int,
                          j_scaling_factor: float, k_scaling_factor: float, d_vj: int, d_vk: int, stream: int = 0):
        """J of dm_s = C_s diag(occ_s) C_s^T and the occupied-orbital K in one
        build (REST generate_hf_hamiltonian_ri_v, scf_io/mod.rs:1339-1381): J's
        aux-row scalars come out of the K half-transform."""
        hm = (C.c_int64 * 2)(*[int(homo[s]) if s < spin_channel else 0 for s in range(2)])
        self._check(lib().rijk_vjk_upper_occ_dev(self._h, C.c_void_p(d_eigv), num_state, hm, C.c_void_p(d_occ),
                                                 spin_channel, float(j_scaling_factor), float(k_scaling_factor),
                                                 C.c_void_p(d_vj), C.c_void_p(d_vk), C.c_void_p(stream or None)))

    def vk_upper_dm_dev(self, d_dm: int, spin_channel: int, scaling_factor: float, d_vk: int, stream: int = 0):
        self._check(lib().rijk_vk_upper_dm_dev(self._h, C.c_void_p(d_dm), spin_channel, float(scaling_factor),
                                               C.c_void_p(d_vk), C.c_void_p(stream or None)))

    # -- MO-basis tensor --------------------------------------------------
    def ao2mo(self, eigv, row_range: range, col_range: range, spin_channel: int = 1):
        """REST ``generate_ri3mo_rayon`` / ``ao2mo_rayon`` (scf_io/mod.rs:2331, :3270):
        per spin an RIFull[N, nrow, ncol] array (Fortran order)."""
        n = self.num_basis
        num_state = np.asarray(eigv[0]).shape[1]
        c = _stack_spin(eigv, spin_channel, (n, num_state))
        nrow, ncol = len(row_range), len(col_range)
        out = np.empty(spin_channel * self.num_auxbas * nrow * ncol)
        self._check(lib().rijk_ao2mo(self._h, _ptr(c), num_state, row_range.start, row_range.stop, col_range.start,
                                     col_range.stop, spin_channel, _ptr(out)))
        per = self.num_auxbas * nrow * ncol
        return [out[s * per:(s + 1) * per].reshape(self.num_auxbas, nrow, ncol, order="F")
                for s in range(spin_channel)]

    # -- split precision (tcgen05) ------------------------------------------
    def vk_upper_occ_split_dev(self, d_eigv: int, num_state: int, homo, d_occ: int, spin_channel: int,
                               scaling_factor: float, d_vk: int, stream: int = 0):
        hm = (C.c_int64 * 2)(*[int(homo[s]) if s < spin_channel else 0 for s in range(2)])
        self._check(lib().rijk_vk_upper_occ_split_dev(self._h, C.c_void_p(d_eigv), num_state, hm, C.c_void_p(d_occ),
                                                      spin_channel, float(scaling_factor), C.c_void_p(d_vk),
                                                      C.c_void_p(stream or None)))

    def vjk_upper_lowrank_split_dev(self, d_v: int, ld_v: int, ncols: int, npos: int, j_scaling_factor: float,
                                    k_scaling_factor: float, accumulate: bool, d_vj: int, d_vk: int,
                                    stream: int = 0):
        """J (overwritten) and K ((+)=) of dD = V S V^T in split precision, J's
        scalars from the split half-transform."""
        self._check(lib().rijk_vjk_upper_lowrank_split_dev(self._h, C.c_void_p(d_v), ld_v, ncols, npos,
                                                           float(j_scaling_factor), float(k_scaling_factor),
                                                           1 if accumulate else 0, C.c_void_p(d_vj),
                                                           C.c_void_p(d_vk), C.c_void_p(stream or None)))

    def vk_upper_lowrank_split_dev(self, d_v: int, ld_v: int, ncols: int, npos: int, scaling_factor: float,
                                   accumulate: bool, d_vk: int, stream: int = 0):
        self._check(lib().rijk_vk_upper_lowrank_split_dev(self._h, C.c_void_p(d_v), ld_v, ncols, npos,
                                                          float(scaling_factor), int(bool(accumulate)),
                                                          C.c_void_p(d_vk), C.c_void_p(stream or None)))

    # -- SCF pieces --------------------------------------------------------
    def density_matrix(self, eigv, homo, occupation, spin_channel: int):
        """REST ``generate_density_matrix`` (scf_io/mod.rs:441): list of n x n D."""
        e0 = np.asarray(eigv[0])
        n, num_state = e0.shape
        c = _stack_spin(eigv, spin_channel, (n, num_state))
        occ = np.ascontiguousarray(np.stack([_f64(occupation[s])[:num_state] for s in range(spin_channel)]))
        hm = (C.c_int64 * 2)(*[int(homo[s]) if s < spin_channel else 0 for s in range(2)])
        out = np.empty(spin_channel * n * n)
        self._check(lib().rijk_density_matrix(self._h, _ptr(c), n, num_state, hm, _ptr(occ), spin_channel, _ptr(out)))
        return [out[s * n * n:(s + 1) * n * n].reshape(n, n, order="F") for s in range(spin_channel)]


GROUP_CFGS = (0, 1, 4)  # CTA shapes the grouped build is compiled for


_GROUP_TILES = {}  # (num_basis, num_auxbas, nocc) -> chosen shapes, for this process


def group_tiles(ctx: "RIJK", nocc: int, sample_rows: int = 256):
    """The project's autotuner applied to a group: times every CTA shape on
    ``ctx``'s tensor (rijk_ctx_autotune) and keeps the fastest of those the
    grouped build supports, for the half-transform and for the rank update.
    The choice is kept per molecule shape for the rest of the process, so that
    repeated runs take the same summation order, and ``ctx``'s own shapes are
    left as they were."""
    key = (*ctx.shape(), int(nocc))
    if key not in _GROUP_TILES:
        before = ctx.tiles()
        _, _, ms = ctx.autotune(int(nocc), int(sample_rows))
        ctx.set_tiles(*before)
        _GROUP_TILES[key] = (min(GROUP_CFGS, key=lambda c: ms[c][0]), min(GROUP_CFGS, key=lambda c: ms[c][1]))
    return _GROUP_TILES[key]


class RIJKGroup:
    """A molecule set's J/K built together (rijk_group_*): one launch per phase
    for every molecule of ``ctxs`` (tensors loaded, left unchanged while the
    group exists)."""

    def __init__(self, ctxs, nocc, half_transform_cfg: int = 1, update_cfg: int = 1):
        self._ctxs = list(ctxs)  # keep the contexts alive
        arr = (C.c_void_p * len(self._ctxs))(*[c.handle.value for c in self._ctxs])
        occ = (C.c_int64 * len(self._ctxs))(*[int(o) for o in nocc])
        h = C.c_void_p()
        st = lib().rijk_group_create(arr, len(self._ctxs), occ, int(half_transform_cfg), int(update_cfg),
                                     C.byref(h))
        if st != 0:
            raise RijkError(st, "cannot create the molecule group")
        self._h = h
        self.tiles = (int(half_transform_cfg), int(update_cfg))

    def jk_occ_dev(self, d_C: int, c_mol: int, c_row: int, c_col: int, k_scale: float, d_active: int, d_out: int,
                   out_mol: int, ldo: int, stream: int = 0):
        st = lib().rijk_group_jk_occ_dev(self._h, C.c_void_p(d_C), int(c_mol), int(c_row), int(c_col),
                                         float(k_scale), C.c_void_p(d_active), C.c_void_p(d_out), int(out_mol),
                                         int(ldo), C.c_void_p(stream or None))
        if st != 0:
            raise RijkError(st, "grouped J/K build failed")

    def synchronize(self, stream: int = 0):
        st = lib().rijk_group_synchronize(self._h, C.c_void_p(stream or None))
        if st != 0:
            raise RijkError(st, "grouped J/K build failed")

    def close(self):
        if getattr(self, "_h", None):
            lib().rijk_group_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 (interpreter shutdown)
            pass


def energy_contraction(a_upper: np.ndarray, b_upper: np.ndarray) -> float:
    """REST ``SCF::par_energy_contraction`` (scf_io/mod.rs:1787)."""
    a = np.ascontiguousarray(_f64(a_upper))
    b = np.ascontiguousarray(_f64(b_upper))
    if a.shape != b.shape:
        raise ValueError("shape mismatch")
    return float(lib().rijk_energy_contraction(_ptr(a), _ptr(b), a.size))
