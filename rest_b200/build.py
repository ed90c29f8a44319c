"""Build librest_b200.so (the C ABI of include/rest_b200.h) in-tree with nvcc.

Every translation unit is compiled for sm_100a only; the library links the
CUDA runtime statically so that the only run-time dependency is the driver.

    python -m rest_b200.build            # build if sources are newer
    python -m rest_b200.build --force    # rebuild
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
BUILD = PKG / "_build"
LIB = PKG / "librest_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "--expt-relaxed-constexpr",
    "-Xcompiler",
    "-fPIC,-O3",
    "-I" + str(INCLUDE),
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build librest_b200.so")


# rijk_ints_cls.cu holds one three-centre integral class, chosen by macros: it is
# compiled once per class (AO l <= 2 twice, auxiliary l <= 4)
INT3C_CLASSES = [(a, b, c) for a in range(3) for b in range(3) for c in range(5)]


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _jobs() -> list[tuple[Path, list[str], str]]:
    """(source, defines, object stem) per object; the per-class integral objects
    first, since their unrolled kernels are the longest compiles."""
    cls, rest = [], []
    for src in sources():
        if src.name == "rijk_ints_cls.cu":
            cls += [(src, [f"-DRIJK_LA={a}", f"-DRIJK_LB={b}", f"-DRIJK_LC={c}"], f"rijk_ints_cls_{a}{b}{c}")
                    for a, b, c in INT3C_CLASSES]
        else:
            rest.append((src, [], src.stem))
    rest.sort(key=lambda j: j[0].stat().st_size, reverse=True)
    return cls + rest


def _stale(lib: Path) -> bool:
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    deps = list(CSRC.glob("*")) + list(INCLUDE.glob("*.h"))
    return any(p.stat().st_mtime > t for p in deps)


def _obj_stale(src: Path, obj: Path) -> bool:
    """An object is rebuilt when its source or any header is newer."""
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))
    return any(p.stat().st_mtime > t for p in [src] + headers)


def _compile(src: Path, extra: list[str], force: bool = False, defines: list[str] | None = None,
             stem: str | None = None) -> Path:
    obj = BUILD / ((stem or src.stem) + ".o")
    if not force and not extra and not _obj_stale(src, obj):
        return obj
    if src.suffix == ".cpp":  # host-only code: g++ with OpenMP
        cmd = ["g++", "-c", str(src), "-o", str(obj), "-O3", "-fPIC", "-fopenmp", "-std=c++17", "-I" + str(INCLUDE)]
    else:
        cmd = [nvcc(), "-c", str(src), "-o", str(obj)] + NVCC_FLAGS + (defines or []) + extra
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
    if os.environ.get("RIJK_PTXAS_VERBOSE"):
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    if not force and not _stale(LIB):
        return LIB
    BUILD.mkdir(exist_ok=True)
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    if verbose_ptxas:
        os.environ["RIJK_PTXAS_VERBOSE"] = "1"
    with cf.ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda j: _compile(j[0], extra, force, j[1], j[2]), _jobs()))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", str(tmp)] + [str(o) for o in objs] + ["-lgomp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose_ptxas=a.ptxas_verbose))


if __name__ == "__main__":
    main()
