"""Extract the basis sets the configs use from REST's basis-set-pool into one
compact JSON per basis (elements H, C, N, O, Cu; exponents, coefficients, l).

The pool is Basis Set Exchange data shipped with REST
(basis-set-pool/<name>/<El>.json); this script is how the committed files in
this directory were made:

    python rest_b200/basis_data/extract.py /path/to/rest/basis-set-pool
"""
import json
import sys
from pathlib import Path

SETS = ["STO-3G", "def2-SVP", "def2-SVP-JKFIT", "def2-SV(P)-JKFIT", "aug-cc-pV5Z"]
ELEMENTS = ["H", "C", "N", "O", "Cu"]


def main(pool: str) -> None:
    out_dir = Path(__file__).resolve().parent
    for name in SETS:
        data = {}
        for el in ELEMENTS:
            f = Path(pool) / name / f"{el}.json"
            if not f.exists():
                continue
            shells = []
            for sh in json.load(open(f))["electron_shells"]:
                ls = sh["angular_momentum"]
                exps = [float(x) for x in sh["exponents"]]
                coefs = [[float(x) for x in col] for col in sh["coefficients"]]
                if len(ls) == 1:
                    for col in coefs:
                        shells.append({"l": ls[0], "exps": exps, "coefs": col})
                else:  # Pople sp shells: one coefficient column per l
                    for l, col in zip(ls, coefs):
                        shells.append({"l": l, "exps": exps, "coefs": col})
            data[el] = shells
        (out_dir / f"{name}.json").write_text(json.dumps(data, separators=(",", ":")))
        print(name, {k: len(v) for k, v in data.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python -m rest_b200.basis_data.extract <REST checkout>/basis-set-pool")
    main(sys.argv[1])
