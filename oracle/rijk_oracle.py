"""CPU FP64 oracle for the RI J/K Fock build: test infrastructure only.

This module restates, in NumPy, the formulas of REST's RI-V Coulomb/exchange
build (jeanwsr/rest, ``src/scf_io/mod.rs``) and of the RI metric step that
produces the fitted three-centre tensor (``src/molecule_io/mod.rs``).  It is the
checker for the CUDA path and nothing else: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` import it.  The
product path (``rest_b200``) never calls into this file.

Parity status: REST has no numerical test for this path (its ``#[test]``
functions only print), and REST itself (Rust, with the unvendored crates
``rest_tensors`` / ``rest_libcint``) cannot be built here.  The restatement is
therefore checked against analytic identities, against a second independent
formulation inside this file (full ``ri3fn`` layout vs packed ``rimatr``,
V^-1/2 metric vs Cholesky metric), and against REST's published example energy
(pentacene RI-HF, ``examples/PEN/RIHF/rest.out``): ``oracle/scf_ctx.py`` runs
the SCF loop on these formulas and ``tests/test_scf_oracle.py`` compares it
with the values in ``tests/golden/pen_rihf.json``.

Storage conventions follow REST (column-major everywhere):

* ``MatrixFull[r, c]``: element (i, j) at ``i + r*j``.  Here a NumPy array with
  ``order='F'`` and shape ``(r, c)``.
* ``MatrixUpper``: packed upper triangle, column by column; (i <= j) at
  ``j*(j+1)/2 + i`` (``molecule_io/mod.rs:731``).
* ``RIFull[n, n, N]``: (mu, nu, P) at ``mu + n*nu + n*n*P``; a NumPy array of
  shape ``(n, n, N)`` with ``order='F'``.
* ``rimatr = MatrixFull[npair, N]``: column P is the packed upper triangle of
  B_P (``molecule_io/mod.rs:1588``, ``:1679-1680``).
"""
from __future__ import annotations

import numpy as np

# ``AUXBAS_THRESHOLD`` (src/constants/mod.rs:81): eigenvalue cut of the metric.
AUXBAS_THRESHOLD = 1.0e-8


# ---------------------------------------------------------------------------
# packed-upper helpers (rest_tensors MatrixUpper semantics)
# ---------------------------------------------------------------------------
def npair_of(n: int) -> int:
    return n * (n + 1) // 2


def upper_pairs(n: int):
    """(i, j) index arrays of the packed upper triangle in REST order.

    REST packs column by column: for j in 0..n, for i in 0..=j
    (``molecule_io/mod.rs:1703-1710`` builds the same map as basbas2baspar).
    """
    jj, ii = np.tril_indices(n)  # rows sorted by jj then ii -> j-major order
    return ii, jj


def to_upper(m: np.ndarray) -> np.ndarray:
    """MatrixFull -> MatrixUpper (keeps the (i<=j) elements)."""
    i, j = upper_pairs(m.shape[0])
    return np.ascontiguousarray(m[i, j])


def from_upper(u: np.ndarray, n: int) -> np.ndarray:
    """MatrixUpper -> symmetric MatrixFull."""
    i, j = upper_pairs(n)
    m = np.zeros((n, n), order="F")
    m[i, j] = u
    m[j, i] = u
    return m


def upper_diag_index(n: int) -> np.ndarray:
    j = np.arange(n)
    return j * (j + 1) // 2 + j


def rimatr_from_ri3fn(ri3fn: np.ndarray) -> np.ndarray:
    """RIFull[n,n,N] -> rimatr [npair, N] (upper triangle of each B_P)."""
    n = ri3fn.shape[0]
    i, j = upper_pairs(n)
    return np.asfortranarray(ri3fn[i, j, :])


def ri3fn_from_rimatr(rimatr: np.ndarray, n: int) -> np.ndarray:
    """rimatr -> RIFull, as ``generate_ri3fn_from_rimatr`` (molecule_io/mod.rs:1723)."""
    naux = rimatr.shape[1]
    i, j = upper_pairs(n)
    out = np.zeros((n, n, naux), order="F")
    out[i, j, :] = rimatr
    out[j, i, :] = rimatr
    return out


# ---------------------------------------------------------------------------
# J builds
# ---------------------------------------------------------------------------
def vj_upper_with_ri_v(ri3fn, dm, spin_channel, scaling_factor):
    """``vj_upper_with_ri_v_sync`` (scf_io/mod.rs:2428-2488).

    Per aux index P: w_P = sum_{mu,nu} B_P[mu,nu] * D[mu,nu] (full n*n dot),
    then J_upper += upper(B_P) * w_P; finally times ``scaling_factor``.
    Returns a list of two packed uppers; the unused spin slot is the
    one-element placeholder REST returns.
    """
    n, _, naux = ri3fn.shape
    out = [np.zeros(1), np.zeros(1)]
    i, j = upper_pairs(n)
    flat = ri3fn.reshape(n * n, naux, order="F")
    for s in range(spin_channel):
        d = np.asarray(dm[s], dtype=np.float64).reshape(n * n, order="F")
        w = flat.T @ d
        out[s] = ri3fn[i, j, :] @ w
    if scaling_factor != 1.0:
        for s in range(spin_channel):
            out[s] = out[s] * scaling_factor
    return out


def vj_upper_with_rimatr_v(rimatr, dm, spin_channel, scaling_factor):
    """``vj_upper_with_rimatr_v_sync`` (scf_io/mod.rs:2490-2561).

    w_P = 2 * sum_{mu<=nu} B[P,mu nu] D_{mu nu} - sum_mu B[P,mu mu] D_{mu mu},
    with D read through its packed upper triangle; J = sum_P B[P,:] w_P.
    """
    npair, naux = rimatr.shape
    n = int(round((np.sqrt(8 * npair + 1) - 1) / 2))
    dg = upper_diag_index(n)
    out = [np.zeros(1), np.zeros(1)]
    for s in range(spin_channel):
        d = np.asarray(dm[s], dtype=np.float64)
        du = to_upper(d)
        w = 2.0 * (rimatr.T @ du) - rimatr[dg, :].T @ np.diag(d)
        out[s] = rimatr @ w
    if scaling_factor != 1.0:
        for s in range(spin_channel):
            out[s] = out[s] * scaling_factor
    return out


def vj_full_with_ri_v(ri3fn, dm, spin_channel, scaling_factor):
    """``vj_full_with_ri_v`` (scf_io/mod.rs:2564-2602): full-matrix J."""
    n, _, naux = ri3fn.shape
    flat = ri3fn.reshape(n * n, naux, order="F")
    out = [np.zeros((1, 1)), np.zeros((1, 1))]
    for s in range(spin_channel):
        d = np.asarray(dm[s], dtype=np.float64).reshape(n * n, order="F")
        w = flat.T @ d
        out[s] = (flat @ w).reshape(n, n, order="F") * scaling_factor
    return out


# ---------------------------------------------------------------------------
# K builds
# ---------------------------------------------------------------------------
def vk_upper_with_ri_v(ri3fn, eigv, homo, occupation, spin_channel, scaling_factor):
    """``vk_upper_with_ri_v_sync`` (scf_io/mod.rs:2758-2834), occupied-orbital form.

    Per P: X = B_P C[:, :nw]; Y = X diag(occ[:nw]); K_P = Y X^T; K_upper += upper(K_P);
    nw = homo + 1.  Then times ``scaling_factor``.
    """
    n, _, naux = ri3fn.shape
    out = [np.zeros(1), np.zeros(1)]
    i, j = upper_pairs(n)
    for s in range(spin_channel):
        nw = homo[s] + 1
        c = np.asarray(eigv[s], dtype=np.float64)[:, :nw]
        occ = np.asarray(occupation[s], dtype=np.float64)[:nw]
        k = np.zeros((n, n))
        for p in range(naux):
            x = ri3fn[:, :, p] @ c
            k += (x * occ) @ x.T
        out[s] = k[i, j]
    if scaling_factor != 1.0:
        for s in range(spin_channel):
            out[s] = out[s] * scaling_factor
    return out


def _symm_from_upper(bp):
    """dsymm with uplo='U' reads only the upper triangle of the symmetric operand."""
    u = np.triu(bp)
    return u + np.triu(bp, 1).T


def vk_upper_with_ri_v_use_dm_only(ri3fn, dm, spin_channel, scaling_factor):
    """``vk_upper_with_ri_v_use_dm_only_sync`` (scf_io/mod.rs:2640-2701).

    Per P: tmp = sym(B_P) D (dsymm 'L','U'); K_P = tmp sym(B_P) (dsymm 'R','U').
    """
    n, _, naux = ri3fn.shape
    out = [np.zeros(1), np.zeros(1)]
    i, j = upper_pairs(n)
    for s in range(spin_channel):
        d = np.asarray(dm[s], dtype=np.float64)
        k = np.zeros((n, n))
        for p in range(naux):
            b = _symm_from_upper(ri3fn[:, :, p])
            k += (b @ d) @ b
        out[s] = k[i, j]
    if scaling_factor != 1.0:
        for s in range(spin_channel):
            out[s] = out[s] * scaling_factor
    return out


def vk_upper_with_rimatr_use_dm_only(rimatr, dm, spin_channel, scaling_factor):
    """``vk_upper_with_rimatr_use_dm_only_sync`` (scf_io/mod.rs:2703-2756).

    Same as the ri3fn dm-only form after unpacking column P of ``rimatr`` into
    the upper triangle of an n*n matrix (``:2726-2728``).
    """
    npair, naux = rimatr.shape
    n = int(round((np.sqrt(8 * npair + 1) - 1) / 2))
    ii, jj = upper_pairs(n)
    out = [np.zeros(1), np.zeros(1)]
    for s in range(spin_channel):
        d = np.asarray(dm[s], dtype=np.float64)
        k = np.zeros((n, n))
        for p in range(naux):
            bu = np.zeros((n, n))
            bu[ii, jj] = rimatr[:, p]
            b = _symm_from_upper(bu)
            k += (b @ d) @ b
        out[s] = k[ii, jj]
    if scaling_factor != 1.0:
        for s in range(spin_channel):
            out[s] = out[s] * scaling_factor
    return out


def vk_full_fromdm_with_ri_v(ri3fn, dm, spin_channel, scaling_factor):
    """``vk_full_fromdm_with_ri_v`` (scf_io/mod.rs:2603-2638).

    Per P: dm_m = D B_P^T (dgemm 'N','T'); K += B_P dm_m.  D may be non-symmetric,
    so the result is a full (possibly non-symmetric) matrix.
    """
    n, _, naux = ri3fn.shape
    out = [np.zeros((1, 1)), np.zeros((1, 1))]
    for s in range(spin_channel):
        d = np.asarray(dm[s], dtype=np.float64)
        k = np.zeros((n, n))
        for p in range(naux):
            b = ri3fn[:, :, p]
            k += b @ (d @ b.T)
        out[s] = k * scaling_factor
    return out


# ---------------------------------------------------------------------------
# RI metric and the fitted tensor (molecule_io/mod.rs:1563-1721)
# ---------------------------------------------------------------------------
def metric_inv_sqrt(v: np.ndarray, threshold: float = AUXBAS_THRESHOLD) -> np.ndarray:
    """``aux_v.lapack_power(-0.5, AUXBAS_THRESHOLD)`` (molecule_io/mod.rs:1582).

    rest_tensors is not vendored, so the semantics are inferred from the call
    site: symmetric eigendecomposition V = U diag(l) U^T, eigenvalues below the
    threshold are discarded, and U_k diag(l_k^-1/2) U_k^T is returned.
    """
    lam, u = np.linalg.eigh(v)
    keep = lam >= threshold
    uk = u[:, keep]
    return np.asfortranarray((uk * lam[keep] ** -0.5) @ uk.T)


def metric_cholesky_factor(v: np.ndarray) -> np.ndarray:
    """Lower Cholesky factor L of V (V = L L^T); raises on a non-SPD metric.

    This is the variant REST keeps commented out beside the live code
    (``cholesky_decompose_inverse('L')``, molecule_io/mod.rs:1583).
    """
    return np.linalg.cholesky(v)


def metric_cholesky_inv_t(v: np.ndarray) -> np.ndarray:
    """M = L^-T, so that M M^T = V^-1; B = (mu nu|Q) M."""
    l = metric_cholesky_factor(v)
    linv = np.linalg.solve(l, np.eye(v.shape[0]))
    return np.asfortranarray(linv.T)


def fit_rimatr(int3c: np.ndarray, m: np.ndarray) -> np.ndarray:
    """rimatr[k, P] = sum_Q int3c[k, Q] M[Q, P]; the per-shell ``_dgemm`` of
    molecule_io/mod.rs:1672-1675 applied to all pairs at once."""
    return np.asfortranarray(int3c @ m)


def fit_rimatr_cholesky(int3c: np.ndarray, v: np.ndarray) -> np.ndarray:
    """B^T = L^-1 (Q|mu nu) by a forward triangular solve (no explicit inverse)."""
    import scipy.linalg as sla

    l = metric_cholesky_factor(v)
    bt = sla.solve_triangular(l, np.ascontiguousarray(int3c.T), lower=True)
    return np.asfortranarray(bt.T)


# ---------------------------------------------------------------------------
# MO-basis three-centre tensor
# ---------------------------------------------------------------------------
def ao2mo(rimatr, eigv, row_range, col_range):
    """``ao2mo_rayon`` (scf_io/mod.rs:3270-3307): per P, tmp = sym(B_P) C (dsymm
    'L','U'), then tmp[:, rows]^T C[:, cols]; stored as RIFull[N, nrow, ncol]."""
    npair, naux = rimatr.shape
    n = int(round((np.sqrt(8 * npair + 1) - 1) / 2))
    ii, jj = upper_pairs(n)
    c = np.asarray(eigv, dtype=np.float64)
    out = np.zeros((naux, len(row_range), len(col_range)), order="F")
    for p in range(naux):
        bu = np.zeros((n, n))
        bu[ii, jj] = rimatr[:, p]
        tmp = _symm_from_upper(bu) @ c
        out[p] = tmp[:, row_range.start:row_range.stop].T @ c[:, col_range.start:col_range.stop]
    return out


# ---------------------------------------------------------------------------
# density, energy, Fock assembly
# ---------------------------------------------------------------------------
def occupation_integer(num_state: int, num_elec_spin: float, occ_num: float):
    """``generate_occupation_integer`` (scf_io/mod.rs:364-440) for one spin."""
    occ = np.zeros(num_state)
    left = float(num_elec_spin)
    idx = 0
    while left > 0.0 and idx <= num_state:
        occ[idx] = min(left * occ_num, occ_num)
        idx += 1
        left -= 1.0
    homo = idx - 1 if idx > 0 else 0
    return occ, homo, idx


def density_matrix(eigv, occupation, homo):
    """``generate_density_matrix`` (scf_io/mod.rs:441-478): D = (C occ) C^T over nw columns."""
    nw = homo + 1
    c = np.asarray(eigv, dtype=np.float64)
    wc = np.zeros_like(c)
    wc[:, :nw] = c[:, :nw] * np.asarray(occupation[:nw])
    return np.asfortranarray(wc @ c.T)


def par_energy_contraction(a_upper, b_upper) -> float:
    """``SCF::par_energy_contraction`` (scf_io/mod.rs:1787-1802):
    1/2 sum_ij a_ij b_ij from packed storage as (2 sum_packed - sum_diag) / 2."""
    n = int(round((np.sqrt(8 * len(a_upper) + 1) - 1) / 2))
    dg = upper_diag_index(n)
    tot = 2.0 * float(np.dot(a_upper, b_upper))
    dc = float(np.dot(a_upper[dg], b_upper[dg]))
    return (tot - dc) * 0.5


def hf_fock_upper(h_core_upper, vj, vk, spin_channel):
    """``generate_hf_hamiltonian_ri_v`` (scf_io/mod.rs:1360-1380): F_s = h + J_0 + J_1 + K_s."""
    fock = []
    for s in range(spin_channel):
        f = h_core_upper.copy()
        if vj[0].size == f.size:
            f = f + vj[0]
        if vj[1].size == f.size:
            f = f + vj[1]
        f = f + vk[s]
        fock.append(f)
    return fock


def hf_energy_rhf(nuc_energy, dm, h_core_upper, fock_upper):
    """RHF total energy (scf_io/mod.rs:1749-1761): E = E_nuc + 1/2 sum D (h + F)."""
    du = to_upper(dm)
    return nuc_energy + par_energy_contraction(du, h_core_upper + fock_upper)
