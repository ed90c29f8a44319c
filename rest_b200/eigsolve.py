"""Warm-started batched symmetric eigensolver for the SCF's Fock matrices.

Between two SCF iterations the orthogonalised Fock matrix X^T F X changes
little, so the previous iteration's eigenvectors are close to the new ones.
Iterative refinement of an approximate eigenbasis (T. Ogita and K. Aishima,
"Iterative refinement for symmetric eigenvalue decomposition", Japan J. Indust.
Appl. Math. 35 (2018) 1007-1035, Algorithm 1) improves such a basis with matrix
products only and converges quadratically.  One refinement step is four batched
n x n FP64 products on the tensor cores, where a fresh eigensolve is a chain of
latency-bound Householder and tridiagonal kernels per molecule.

Step, for A symmetric and V an approximate orthonormal eigenbasis:

    R = I - V^T V,  S = V^T A V,  lam_i = s_ii / (1 - r_ii)
    e_ij = (s_ij + lam_j r_ij) / (lam_j - lam_i)   (i != j; clipped, below)
    e_ii = r_ii / 2
    V <- V + V E

The paper treats pairs closer than one global bound on the eigenvalue error as
a cluster (e_ij = r_ij / 2, no rotation); on the orthogonalised Fock matrices of
water clusters that leaves near-degenerate pairs (the waters' O 1s and valence
levels) unrotated for good, and the refinement stalls while the Fock matrix
still moves by 1e-2..1e-1 Eh between iterations.  Here every off-diagonal e_ij
takes the first-order value clipped to [-1/4, 1/4]: a strongly coupled close
pair turns by a bounded step in the right direction, the next step sees it
better separated, and the usual quadratic convergence follows (measured on the
SCF sequences of (H2O)4 and (H2O)8 in def2-SVP: from a Fock change of 0.1 Eh to
eigenvalues within 4e-14 Eh in at most 8 steps).  A molecule passes when, after
the last step, the off-diagonal of V^T A V (for an orthonormal V, the residual
A V - V Lam) is at most ``tol_off`` times max(1, max |lam|) and V^T V is the
identity to ``tol_orth``; the caller diagonalises the others from scratch.
Steps from a basis that is too far off diverge (to inf / NaN), which the same
check rejects.

Padded batches: molecule b uses the leading ``nvalid[b]`` rows and columns; the
padded block of A must be a multiple of the identity decoupled from the rest
and the padded block of V the identity, which every step leaves unchanged
(their rotations are zero).  Eigenvalues come back in ascending order with the
padding last.
"""
from __future__ import annotations


def _pair_mask(torch, nvalid, nm, device):
    ar = torch.arange(nm, device=device)
    valid = ar[None, :] < nvalid[:, None]  # B x nm
    return valid[:, :, None] & valid[:, None, :]


def _gram(torch, A, V, nm):
    """G = V^T V and S = V^T A V from one product, symmetrised: the rounding
    asymmetry of S (about n eps |A|) divided by a close pair's gap would
    otherwise become an orthogonality error of the update."""
    GS = V.transpose(1, 2) @ torch.cat([V, A @ V], dim=2)
    G, S = GS[:, :, :nm], GS[:, :, nm:]
    return 0.5 * (G + G.transpose(1, 2)), 0.5 * (S + S.transpose(1, 2))


def refine(A, V, nvalid, steps: int = 4, tol_off: float = 1e-10, tol_orth: float = 1e-10,
           clip: float = 0.25):
    """Refine the batched eigenbases V (B x nm x nm, columns = vectors) of the
    symmetric A.  Returns (lam, V, ok, off): eigenvalues ascending, the refined
    and reordered vectors, a bool per molecule that says whether it passed, and
    the largest off-diagonal of V^T A V relative to max(1, max |lam|)."""
    import torch

    B, nm, _ = A.shape
    dev = A.device
    nvalid = torch.as_tensor(nvalid, device=dev)
    pairs = _pair_mask(torch, nvalid, nm, dev)
    eye = torch.eye(nm, dtype=A.dtype, device=dev)
    offd = pairs & ~eye.bool()[None]
    for _ in range(steps):
        G, S = _gram(torch, A, V, nm)
        R = eye - G
        lam = torch.diagonal(S, dim1=1, dim2=2) / torch.diagonal(G, dim1=1, dim2=2)
        num = S + lam[:, None, :] * R
        gap = lam[:, None, :] - lam[:, :, None]
        # first-order rotation num / gap, clipped; a zero gap takes the clip's sign of num
        t = torch.where(num.abs() < clip * gap.abs(), num / torch.where(gap == 0, torch.ones_like(gap), gap),
                        clip * torch.sign(num) * torch.where(gap < 0, -1.0, 1.0))
        E = torch.where(offd, t, torch.where(pairs, 0.5 * R, torch.zeros_like(R)))
        V = V + V @ E
    G, S = _gram(torch, A, V, nm)
    lam = torch.diagonal(S, dim1=1, dim2=2) / torch.diagonal(G, dim1=1, dim2=2)
    valid = torch.arange(nm, device=dev)[None, :] < nvalid[:, None]
    scale = torch.where(valid, lam.abs(), torch.zeros_like(lam)).amax(dim=1).clamp(min=1.0)
    off = torch.where(offd, S.abs(), torch.zeros_like(S)).amax(dim=(1, 2)) / scale
    orth = torch.where(pairs, (G - eye).abs(), torch.zeros_like(G)).amax(dim=(1, 2))
    ok = (off <= tol_off) & (orth <= tol_orth)  # NaN compares false
    order = torch.argsort(torch.where(valid, lam, torch.full_like(lam, float("inf"))), dim=1, stable=True)
    lam = torch.gather(lam, 1, order)
    V = torch.gather(V, 2, order[:, None, :].expand(B, nm, nm))
    return lam, V, ok, off


def eigh_batched(A, nvalid, pad_value: float = 1.0e6):
    """All eigenpairs of the symmetric matrices A (B x nm x nm, FP64, device) with
    the library's batched solver (rijk_eigh_batched_dev: Householder
    tridiagonalisation and implicit QL, one CTA per matrix).  Matrix b uses its
    leading nvalid[b] rows and columns; the padding gets eigenvalue pad_value and
    unit vectors.  Returns (lam ascending, V with vectors as columns, ok per
    matrix); A is not modified."""
    import ctypes as C

    import torch

    from ._abi import RijkError, lib

    B, nm, _ = A.shape
    dev = A.device
    a = A.contiguous().clone()
    nv = torch.as_tensor(list(nvalid), dtype=torch.int32, device=dev)
    lam = torch.empty(B, nm, dtype=A.dtype, device=dev)
    V = torch.empty(B, nm, nm, dtype=A.dtype, device=dev)
    work = torch.empty(B, nm, nm, dtype=A.dtype, device=dev)
    info = torch.empty(B, dtype=torch.int32, device=dev)
    st = lib().rijk_eigh_batched_dev(C.c_void_p(a.data_ptr()), nm, C.c_void_p(nv.data_ptr()), B, float(pad_value),
                                     C.c_void_p(lam.data_ptr()), C.c_void_p(V.data_ptr()),
                                     C.c_void_p(work.data_ptr()), C.c_void_p(info.data_ptr()),
                                     C.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    if st != 0:
        raise RijkError(st, "batched eigensolver")
    return lam, V, info == 0


def diis_coefficients(gram, count):
    """REST's diis_solver for a batch (rijk_diis_coefficients_dev): gram is
    B x m x m (FP64, device), count[b] the history length of molecule b (its
    leading min(count, m) slots are used).  Returns (coef B x m, failed B bool):
    a molecule whose Gram matrix is exactly singular gets (1, 0, ..., 0) and
    failed = True, and its caller restarts the history from slot 0."""
    import ctypes as C

    import torch

    from ._abi import RijkError, lib

    B, m, _ = gram.shape
    dev = gram.device
    g = gram.contiguous()
    cnt = torch.as_tensor(count, dtype=torch.int32, device=dev)
    coef = torch.empty(B, m, dtype=torch.float64, device=dev)
    status = torch.empty(B, dtype=torch.int32, device=dev)
    st = lib().rijk_diis_coefficients_dev(C.c_void_p(g.data_ptr()), m, C.c_void_p(cnt.data_ptr()), B,
                                          C.c_void_p(coef.data_ptr()), C.c_void_p(status.data_ptr()),
                                          C.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    if st != 0:
        raise RijkError(st, "batched DIIS coefficients")
    return coef, status != 0
