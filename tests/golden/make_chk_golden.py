"""Copy the smallest libhdf5-written file of REST's examples into tests/golden.

REST exchanges guess densities and orbitals through HDF5 files
(src/initial_guess/mod.rs:71-124).  REST's repository ships several such files
written by libhdf5 (through PySCF/h5py); the smallest,
examples/Cu2/HF_SAD/init_guess.chk (148 KB: datasets init_guess, mol and the
group scf with e_tot, mo_coeff, mo_energy, mo_occ for Cu2 in def2-SVP, n = 62),
is copied unchanged as tests/golden/cu2_init_guess.chk, and its geometry
(examples/Cu2/HF_SAD/ctrl.in) and SHA-256 go to tests/golden/cu2_chk.json.
tests/test_chkfile.py reads it with rest_b200.chkfile (no libhdf5 here).

    python tests/golden/make_chk_golden.py <REST checkout>
"""
import hashlib
import json
import shutil
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_chk_golden.py <REST checkout>")
    d = Path(sys.argv[1]) / "examples" / "Cu2" / "HF_SAD"
    src = d / "init_guess.chk"
    dst = HERE / "cu2_init_guess.chk"
    shutil.copyfile(src, dst)
    ctrl = (d / "ctrl.in").read_text()
    block = ctrl.split("position = '''")[1].split("'''")[0]
    symbols, coords = [], []
    for line in block.strip().splitlines():
        p = line.split()
        symbols.append(p[0])
        coords.append([float(v) for v in p[1:4]])
    out = {
        "source": "REST examples/Cu2/HF_SAD: init_guess.chk (written by libhdf5 through PySCF), ctrl.in",
        "symbols": symbols,
        "coords_angstrom": coords,
        "basis": "def2-SVP",
        "num_basis": 62,
        "nelec": 58,
        "sha256": hashlib.sha256(dst.read_bytes()).hexdigest(),
    }
    (HERE / "cu2_chk.json").write_text(json.dumps(out, indent=1))
    print("wrote", dst, HERE / "cu2_chk.json")


if __name__ == "__main__":
    main()
