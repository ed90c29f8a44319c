"""CPU stand-in for rest_b200.RIJK built from the oracle (test infrastructure).

It offers the methods rest_b200.scf.SCF calls on a device context, computed
with the NumPy restatement of REST's formulas, so that the same SCF loop runs
entirely on the CPU oracle.  Used by tests to pin the SCF driver against
REST's published energies and to compare the GPU path with the oracle.
"""
from __future__ import annotations

import numpy as np

from . import rijk_oracle as O


class OracleRIJK:
    def __init__(self):
        self.rimatr = None
        self.num_basis = 0

    def spawn(self):
        return OracleRIJK()

    def fit_rimatr(self, metric_factor, int3c, num_basis):
        self.rimatr = O.fit_rimatr(np.asfortranarray(int3c), np.asarray(metric_factor))
        self.num_basis = num_basis

    def build_rimatr_cholesky(self, aux_v, int3c, num_basis):
        self.rimatr = O.fit_rimatr_cholesky(np.asfortranarray(int3c), np.asarray(aux_v))
        self.num_basis = num_basis

    def set_rimatr(self, rimatr, num_basis):
        self.rimatr = np.asfortranarray(rimatr)
        self.num_basis = num_basis

    def vj_upper_with_rimatr_v(self, dm, spin_channel, scale):
        return O.vj_upper_with_rimatr_v(self.rimatr, dm, spin_channel, scale)

    def vj_upper_with_ri_v(self, dm, spin_channel, scale):
        return O.vj_upper_with_rimatr_v(self.rimatr, [0.5 * (d + d.T) for d in dm[:spin_channel]], spin_channel,
                                        scale)

    def vk_upper_with_rimatr_use_dm_only(self, dm, spin_channel, scale):
        return self._vk_dm(dm, spin_channel, scale)

    def vk_upper_with_ri_v_use_dm_only(self, dm, spin_channel, scale):
        return self._vk_dm(dm, spin_channel, scale)

    def _vk_dm(self, dm, spin_channel, scale):
        # batched over P: K = sum_P B_P D B_P, same arithmetic as the per-P oracle loop
        n = self.num_basis
        ii, jj = O.upper_pairs(n)
        out = [np.zeros(1), np.zeros(1)]
        naux = self.rimatr.shape[1]
        for s in range(spin_channel):
            d = np.asarray(dm[s])
            k = np.zeros((n, n))
            for p0 in range(0, naux, 64):
                p1 = min(naux, p0 + 64)
                b = np.zeros((p1 - p0, n, n))
                b[:, ii, jj] = self.rimatr[:, p0:p1].T
                b[:, jj, ii] = self.rimatr[:, p0:p1].T
                k += np.einsum("pij,pjk->ik", b @ d, b, optimize=True)
            out[s] = k[ii, jj] * scale
        return out

    def vk_upper_with_ri_v(self, eigv, homo, occupation, spin_channel, scale):
        dm = [O.density_matrix(eigv[s], occupation[s], homo[s]) for s in range(spin_channel)]
        return self._vk_dm(dm, spin_channel, scale)

    def density_matrix(self, eigv, homo, occupation, spin_channel):
        return [O.density_matrix(eigv[s], occupation[s], homo[s]) for s in range(spin_channel)]
