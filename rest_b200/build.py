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


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


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


def _compile(src: Path, extra: list[str], force: bool = False) -> Path:
    obj = BUILD / (src.stem + ".o")
    if not force and not extra and not _obj_stale(src, obj):
        return obj
    if src.suffix == ".cpp":  # host-only code: g++ with OpenMP
        cmd = ["g++", "-c", str(src), "-o", str(obj), "-O3", "-fPIC", "-fopenmp", "-std=c++17", "-I" + str(INCLUDE)]
    else:
        cmd = [nvcc(), "-c", str(src), "-o", str(obj)] + NVCC_FLAGS + extra
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
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        # longest compiles first so that they overlap the short ones
        srcs = sorted(sources(), key=lambda p: p.stat().st_size, reverse=True)
        objs = list(ex.map(lambda s: _compile(s, extra, force), srcs))
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
