"""Seeded synthetic RI-JK inputs (the FP64 kernel-sweep workload).

Workload definition (n = num_basis, N = num_auxbas = 4n, o = nocc = n // 6):
  * AO centres r_mu uniform in a 20 Angstrom cube;
  * s_P log-uniform in [1e-3, 1];
  * B[P, mu<=nu] = s_P * exp(-0.1 |r_mu - r_nu|^2) * N(0, 1), stored packed in
    REST's rimatr layout (MatrixFull[npair, N], column P = upper triangle of B_P);
  * C_occ = Q of the QR factorisation of an N(0,1) n x o matrix; D = C_occ C_occ^T.

``host_case`` draws everything with NumPy (used for parity tests, where the
same arrays go to the oracle and to the device).  ``device_case`` draws the
same distributions with torch's CUDA generator straight into the device tensor
in row chunks (used for the full-size benchmark, where a host copy of a 28 GB
tensor would dominate); its numbers differ from the NumPy draw.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class SynthCase:
    n: int
    naux: int
    nocc: int
    seed: int
    rimatr: np.ndarray | None  # [npair, naux] Fortran (None for device cases)
    c_occ: np.ndarray  # [n, nocc] Fortran
    dm: np.ndarray  # [n, n] Fortran

    @property
    def npair(self) -> int:
        return self.n * (self.n + 1) // 2


def sweep_sizes(n: int) -> tuple[int, int, int]:
    return n, 4 * n, n // 6


def _pairs(n: int):
    jj, ii = np.tril_indices(n)
    return ii, jj  # REST packed-upper order: column j, rows i <= j


def host_case(n: int, naux: int | None = None, nocc: int | None = None, seed: int = 2024,
              rows: tuple[int, int] | None = None) -> SynthCase:
    """NumPy draw.  ``rows=(p0, p1)`` keeps only aux rows [p0, p1) of B (the
    full-row draw order is preserved, so a sample equals the same rows of the
    full tensor)."""
    _, n4, n6 = sweep_sizes(n)
    naux = n4 if naux is None else naux
    nocc = max(1, n6) if nocc is None else nocc
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.0, 20.0, size=(n, 3))
    s = np.exp(rng.uniform(math.log(1e-3), math.log(1.0), size=naux))
    c = np.linalg.qr(rng.standard_normal((n, nocc)))[0]
    ii, jj = _pairs(n)
    d2 = np.sum((r[ii] - r[jj]) ** 2, axis=1)
    env = np.exp(-0.1 * d2)
    npair = ii.size
    p0, p1 = (0, naux) if rows is None else rows
    b = np.empty((p1 - p0, npair))
    brng = np.random.default_rng([seed, 1])
    if p0 > 0:
        brng.standard_normal((p0, npair))  # advance the stream to row p0
    for p in range(p0, p1):
        b[p - p0] = brng.standard_normal(npair) * (s[p] * env)
    c_occ = np.asfortranarray(c)
    dm = np.asfortranarray(c_occ @ c_occ.T)
    return SynthCase(n, naux, nocc, seed, np.asfortranarray(b.T), c_occ, dm)


def device_case(ctx, n: int, naux: int | None = None, nocc: int | None = None, seed: int = 2024,
                chunk_bytes: int = 1 << 30):
    """Fill ``ctx`` (a ``rest_b200.RIJK``) with a device-drawn tensor; returns
    (c_occ, dm) as CUDA float64 torch tensors (column-major storage, i.e. the
    transposed row-major tensors)."""
    import torch

    _, n4, n6 = sweep_sizes(n)
    naux = n4 if naux is None else naux
    nocc = max(1, n6) if nocc is None else nocc
    dev = torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    f64 = torch.float64
    r = torch.rand(n, 3, generator=g, dtype=f64, device=dev) * 20.0
    lo, hi = math.log(1e-3), 0.0
    s = torch.exp(lo + (hi - lo) * torch.rand(naux, generator=g, dtype=f64, device=dev))
    c = torch.linalg.qr(torch.randn(n, nocc, generator=g, dtype=f64, device=dev))[0]
    ii, jj = (torch.as_tensor(a, device=dev) for a in _pairs(n))
    env = torch.exp(-0.1 * ((r[ii] - r[jj]) ** 2).sum(dim=1))
    npair = ii.numel()
    ctx.tensor_alloc(n, naux)
    rows = max(1, min(naux, chunk_bytes // (npair * 8)))
    stream = torch.cuda.current_stream().cuda_stream
    buf = torch.empty(rows, npair, dtype=f64, device=dev)
    for p0 in range(0, naux, rows):
        np_ = min(rows, naux - p0)
        torch.randn(np_, npair, generator=g, dtype=f64, device=dev, out=buf[:np_])
        buf[:np_].mul_(s[p0:p0 + np_, None]).mul_(env[None, :])
        ctx.tensor_load_rows_dev(buf.data_ptr(), p0, np_, 0, stream)
    torch.cuda.synchronize()
    del buf
    c_cm = c.t().contiguous()  # column-major n x o  ==  row-major o x n
    dm = (c @ c.t()).contiguous()  # symmetric: row-major == column-major
    return c_cm, dm
