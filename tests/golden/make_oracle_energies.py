"""Converged RI-HF energies on the CPU oracle for the application configs.

The molecule-set and precision configs report their energy errors against the
FP64 oracle.  Converging the oracle SCF takes minutes per molecule on the
host, so the energies of a fixed subset are computed once here and committed
as tests/golden/oracle_energies.json; bench.py reads that file (it never runs
the oracle for these configs) and tests/test_golden_energies.py recomputes
the smallest entry on every CPU test run.

  water_set   clusters 0, 2, 4, 9, 21 of the seeded water-cluster set
              (rest_b200.geometry.water_cluster_set_spec, seed 2024; k = 4, 2,
              6, 16, 10): def2-SVP / def2-SVP-JKFIT, RHF, Cholesky metric (the
              batched driver's), host integrals.
  alkanes     C10H22, same basis and metric.

Each SCF runs rest_b200.scf's restatement of REST's loop on the oracle's J/K
(oracle/scf_ctx.py) to |dE| <= 1e-10 Eh.

    python tests/golden/make_oracle_energies.py
"""
import json
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

SET_SEED = 2024
SET_INDICES = (0, 2, 4, 9, 21)
BASIS, AUXBAS = "def2-SVP", "def2-SVP-JKFIT"


def oracle_energy(mol) -> dict:
    from oracle.scf_ctx import OracleRIJK
    from rest_b200.scf import SCF, ScfOptions

    opts = ScfOptions(metric="cholesky", integrals="host", scf_acc_etot=1e-10, scf_acc_rho=1e-8,
                      scf_acc_eev=1e-8, max_scf_cycle=200)
    t0 = time.perf_counter()
    r = SCF(mol, BASIS, AUXBAS, opts, ctx=OracleRIJK()).run()
    if not r.converged:
        raise RuntimeError("oracle SCF did not converge")
    return {"energy": r.energy, "iterations": r.iterations, "num_basis": r.num_basis, "num_auxbas": r.num_auxbas,
            "oracle_s": round(time.perf_counter() - t0, 1)}


def main():
    from rest_b200.geometry import alkane, water_cluster, water_cluster_set_spec

    spec = water_cluster_set_spec(max(SET_INDICES) + 1, SET_SEED)
    out = {"basis": BASIS, "auxbas": AUXBAS, "metric": "cholesky", "convergence_etot": 1e-10,
           "water_set": {"seed": SET_SEED, "entries": []}, "alkanes": []}
    for i in SET_INDICES:
        k, seed = spec[i]
        rec = {"index": i, "k": k, "seed": seed, **oracle_energy(water_cluster(k, seed))}
        print(rec, flush=True)
        out["water_set"]["entries"].append(rec)
    for nc in (10,):
        rec = {"molecule": f"C{nc}H{2 * nc + 2}", "carbons": nc, **oracle_energy(alkane(nc))}
        print(rec, flush=True)
        out["alkanes"].append(rec)
    (HERE / "oracle_energies.json").write_text(json.dumps(out, indent=1))
    print("wrote", HERE / "oracle_energies.json")


if __name__ == "__main__":
    main()
