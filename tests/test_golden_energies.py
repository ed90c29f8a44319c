"""The committed oracle energies of the application configs are reproducible.

tests/golden/oracle_energies.json holds FP64 CPU-oracle RI-HF energies of a
fixed subset of the seeded water-cluster set and of C10H22
(tests/golden/make_oracle_energies.py); bench.py reports the batched and
mixed-precision energies against them.  Here the subset's indices must still
name the same clusters, and the smallest cluster is converged again on the
oracle and must give the committed energy.
"""
import json
from pathlib import Path

from oracle.scf_ctx import OracleRIJK
from rest_b200.geometry import water_cluster, water_cluster_set_spec
from rest_b200.scf import SCF, ScfOptions

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "oracle_energies.json").read_text())


def test_subset_names_the_same_clusters():
    ws = GOLDEN["water_set"]
    spec = water_cluster_set_spec(512, ws["seed"])
    for e in ws["entries"]:
        assert tuple(spec[e["index"]]) == (e["k"], e["seed"])
        assert e["num_basis"] == 24 * e["k"] and e["num_auxbas"] == 113 * e["k"]


def test_smallest_cluster_energy_reproduces():
    e = min(GOLDEN["water_set"]["entries"], key=lambda x: x["k"])
    opts = ScfOptions(metric="cholesky", integrals="host", scf_acc_etot=1e-10, scf_acc_rho=1e-8, scf_acc_eev=1e-8,
                      max_scf_cycle=200)
    r = SCF(water_cluster(e["k"], e["seed"]), GOLDEN["basis"], GOLDEN["auxbas"], opts, ctx=OracleRIJK()).run()
    assert r.converged
    assert abs(r.energy - e["energy"]) < 1e-9
