"""GPU-resident batched RI-HF (rest_b200.scf_batch) against the per-molecule SCF.

The batch advances water clusters of uneven size together (device J/K per
molecule on its own stream, device Fock/DIIS/eigensolve on the padded batch);
every converged energy must equal the single-molecule driver's FP64 energy.
"""
import pytest

from rest_b200.scf import SCF, ScfOptions
from rest_b200.scf_batch import BatchedRHF, water_cluster

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-8), ("split", 2e-4)])
def test_batched_water_clusters_match_single_scf(ctx, precision, tol):
    mols = [water_cluster(k, seed=10 + k) for k in (1, 2, 3, 1, 2)]
    batch = BatchedRHF(mols, "def2-SVP", "def2-SVP-JKFIT", precision=precision)
    # all-split builds carry ~1e-5 relative noise in K: converge them loosely
    crit = dict(acc_etot=1e-10, acc_rho=1e-7, acc_eev=1e-7) if precision == "fp64" else \
        dict(acc_etot=1e-5, acc_rho=1e-4, acc_eev=1e-3)
    try:
        res = batch.run(max_cycle=100, **crit)
    finally:
        batch.close()
    assert all(res.converged)
    opts = ScfOptions(use_ri_symm=False, scf_acc_etot=1e-10, scf_acc_rho=1e-7, scf_acc_eev=1e-7, max_scf_cycle=100)
    for mol, e in zip(mols, res.energies):
        ref = SCF(mol, "def2-SVP", "def2-SVP-JKFIT", opts, ctx=ctx).run()
        assert ref.converged
        # split-precision K (no FP64 finish in the batch) keeps ~1e-5 relative accuracy
        assert abs(e - ref.energy) < tol * (1.0 if precision == "fp64" else abs(ref.energy))
