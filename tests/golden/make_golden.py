"""Generate the golden fixtures of tests/golden from REST's example run and the oracle.

REST cannot be built here, and its own tests assert no J/K or energy value;
the values REST itself published for this path are the example logs beside
its inputs.  This script extracts them, so that tests never read REST's tree:

  pen_rihf.json   pentacene RI-HF (STO-3G / def2-SV(P)-JKFIT, RHF, use_ri_symm):
                  geometry from examples/PEN/RIHF/ctrl.in, and from
                  examples/PEN/RIHF/rest.out the nuclear repulsion
                  ("Nuc_energy:"), the lowest overlap eigenvalue ("Lowest
                  eigenvalue:"), basis sizes ("numbasis: ..., num_auxbas: ...")
                  and the converged energy (last "Energy:" line); PySCF's
                  energy from rihf_pen.pyscf.log ("converged SCF energy").
  water_rihf.json water RI-HF (def2-SVP / def2-SVP-JKFIT, RHF) converged with the
                  CPU oracle (no REST log exists for it): the reference the GPU
                  SCF must reproduce within 1e-9 Eh.
  nh3_dimer_cation_rihf.json
                  (NH3)2+ RI-UHF (aug-cc-pV5Z / def2-SV(P)-JKFIT, doublet,
                  use_ri_symm and use_dm_only): geometry, charge and spin from
                  examples/RIHF-NH3-dimer/ctrl.in, basis sizes and the last
                  "Energy:" line of its rest.out, PySCF's energy from its
                  pyscf.log, and the energy of the CPU oracle's SCF from the same
                  input (about four minutes on eight cores).

    python tests/golden/make_golden.py /path/to/rest
"""
import json
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))


def pen(rest: Path) -> dict:
    d = rest / "examples" / "PEN" / "RIHF"
    ctrl = (d / "ctrl.in").read_text()
    block = ctrl.split("position = '''")[1].split("'''")[0]
    symbols, coords = [], []
    for line in block.strip().splitlines():
        p = line.split()
        symbols.append(p[0])
        coords.append([float(v) for v in p[1:4]])
    out = (d / "rest.out").read_text()
    enuc = float(re.search(r"Nuc_energy:\s*([-\d.eE+]+)", out).group(1))
    lowest = float(re.search(r"Lowest eigenvalue:\s*([-\d.eE+]+)", out).group(1))
    nb = re.search(r"numbasis:\s*(\d+), num_auxbas:\s*(\d+)", out)
    energies = re.findall(r"Energy:\s*([-\d.]+) Ha after\s+(\d+) iterations", out)
    e_last, it_last = energies[-1]
    py = (d / "rihf_pen.pyscf.log").read_text()
    e_py = float(re.search(r"converged SCF energy = ([-\d.]+)", py).group(1))
    return {
        "source": "REST examples/PEN/RIHF: ctrl.in (geometry, keys), rest.out, rihf_pen.pyscf.log",
        "symbols": symbols,
        "coords_angstrom": coords,
        "basis": "STO-3G",
        "auxbas": "def2-SV(P)-JKFIT",
        "ctrl": {"use_ri_symm": True, "use_dm_only": False, "mixer": "diis", "num_max_diis": 8,
                 "start_diis_cycle": 1, "mix_param": 0.6, "scf_acc_rho": 1e-5, "scf_acc_eev": 1e-5,
                 "scf_acc_etot": 1e-8},
        "rest_nuc_energy": enuc,
        "rest_ovlp_lowest_eigenvalue": lowest,
        "rest_num_basis": int(nb.group(1)),
        "rest_num_auxbas": int(nb.group(2)),
        "rest_energy": float(e_last),
        "rest_iterations": int(it_last),
        "pyscf_energy": e_py,
    }


def water() -> dict:
    from oracle.scf_ctx import OracleRIJK
    from rest_b200.basis import Molecule
    from rest_b200.scf import SCF, ScfOptions

    symbols = ["O", "H", "H"]
    coords = [[0.0, 0.0, 0.0], [0.757, 0.587, 0.0], [-0.757, 0.587, 0.0]]
    mol = Molecule.from_angstrom(symbols, coords)
    opts = ScfOptions(scf_acc_etot=1e-11, scf_acc_rho=1e-8, scf_acc_eev=1e-8, max_scf_cycle=200)
    r = SCF(mol, "def2-SVP", "def2-SVP-JKFIT", opts, ctx=OracleRIJK()).run()
    return {
        "source": "CPU oracle (oracle/rijk_oracle.py via oracle/scf_ctx.py), rest_b200.basis integrals",
        "symbols": symbols,
        "coords_angstrom": coords,
        "basis": "def2-SVP",
        "auxbas": "def2-SVP-JKFIT",
        "num_basis": r.num_basis,
        "num_auxbas": r.num_auxbas,
        "oracle_energy": r.energy,
        "oracle_iterations": r.iterations,
        "nuc_energy": r.nuc_energy,
    }


def nh3_dimer_cation(rest: Path) -> dict:
    from oracle.scf_ctx import OracleRIJK
    from rest_b200.basis import Molecule
    from rest_b200.scf import SCF, ScfOptions

    d = rest / "examples" / "RIHF-NH3-dimer"
    ctrl = (d / "ctrl.in").read_text()
    block = ctrl.split("position = '''")[1].split("'''")[0]
    symbols, coords = [], []
    for line in block.strip().splitlines():
        p = line.split()
        symbols.append(p[0])
        coords.append([float(v) for v in p[1:4]])
    charge = int(float(re.search(r"charge\s*=\s*([-\d.]+)", ctrl).group(1)))
    spin = int(float(re.search(r"\bspin\s*=\s*([-\d.]+)", ctrl).group(1)))
    out = (d / "rest.out").read_text()
    nb = re.search(r"numbasis:\s*(\d+), num_auxbas:\s*(\d+)", out)
    energies = re.findall(r"Energy:\s*([-\d.]+) Ha after\s+(\d+) iterations", out)
    e_last, it_last = energies[-1]
    py = (d / "pyscf.log").read_text()
    e_py = float(re.search(r"converged SCF energy = ([-\d.]+)", py).group(1))
    mol = Molecule.from_angstrom(symbols, coords, charge=charge, spin=spin)
    opts = ScfOptions(use_ri_symm=True, use_dm_only=True)
    r = SCF(mol, "aug-cc-pV5Z", "def2-SV(P)-JKFIT", opts, ctx=OracleRIJK()).run()
    return {
        "source": "REST examples/RIHF-NH3-dimer: ctrl.in (geometry, charge, spin, keys), rest.out, pyscf.log; "
                  "oracle_energy: CPU oracle (oracle/rijk_oracle.py via oracle/scf_ctx.py)",
        "symbols": symbols,
        "coords_angstrom": coords,
        "charge": charge,
        "spin": spin,
        "basis": "aug-cc-pV5Z",
        "auxbas": "def2-SV(P)-JKFIT",
        "ctrl": {"use_ri_symm": True, "use_dm_only": True, "mixer": "diis", "num_max_diis": 8,
                 "start_diis_cycle": 1, "mix_param": 0.6, "scf_acc_rho": 1e-5, "scf_acc_eev": 1e-5,
                 "scf_acc_etot": 1e-8, "initial_guess_rest": "sad"},
        "rest_num_basis": int(nb.group(1)),
        "rest_num_auxbas": int(nb.group(2)),
        "rest_energy": float(e_last),
        "rest_iterations": int(it_last),
        "pyscf_energy": e_py,
        "oracle_energy": r.energy,
        "oracle_iterations": r.iterations,
    }


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <REST checkout>")
    rest = Path(sys.argv[1])
    (HERE / "pen_rihf.json").write_text(json.dumps(pen(rest), indent=1))
    (HERE / "water_rihf.json").write_text(json.dumps(water(), indent=1))
    (HERE / "nh3_dimer_cation_rihf.json").write_text(json.dumps(nh3_dimer_cation(rest), indent=1))
    print("wrote", HERE / "pen_rihf.json", HERE / "water_rihf.json", HERE / "nh3_dimer_cation_rihf.json")


if __name__ == "__main__":
    main()
