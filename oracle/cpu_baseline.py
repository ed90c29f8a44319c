"""Timed CPU baseline: REST's RI J/K algorithm restated in C (oracle/cpu_rijk.c).

Test and benchmark infrastructure only.  ``build()`` compiles the C file with
gcc/OpenMP into oracle/_build; ``CpuRijk`` binds it with ctypes and points it
at the OpenBLAS that ships inside NumPy (ILP64, ``scipy_`` symbols).
"""
from __future__ import annotations

import ctypes as C
import glob
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "cpu_rijk.c"
LIB = HERE / "_build" / "libcpu_rijk.so"


def openblas_path() -> str:
    base = Path(np.__file__).resolve().parent.parent / "numpy.libs"
    cands = sorted(glob.glob(str(base / "libscipy_openblas64_*.so")))
    if not cands:
        raise RuntimeError(f"no scipy-openblas library under {base}")
    return cands[0]


def build(force: bool = False) -> Path:
    if LIB.exists() and not force and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    LIB.parent.mkdir(exist_ok=True)
    tmp = LIB.with_suffix(".tmp.so")
    cmd = ["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", str(SRC), "-o", str(tmp), "-ldl"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


class CpuRijk:
    def __init__(self, nthreads: int | None = None):
        L = C.CDLL(str(build()))
        L.cpu_rijk_init.argtypes = [C.c_char_p]
        if L.cpu_rijk_init(openblas_path().encode()) != 0:
            raise RuntimeError("cannot bind OpenBLAS")
        vp, i64, d = C.c_void_p, C.c_int64, C.c_double
        L.cpu_vj_upper_with_rimatr.argtypes = [vp, i64, i64, vp, d, C.c_int, vp]
        L.cpu_vk_upper_with_ri_v.argtypes = [vp, i64, i64, vp, i64, i64, vp, d, C.c_int, vp]
        self.L = L
        self.nthreads = int(nthreads or os.cpu_count() or 1)

    def vj_upper_with_rimatr(self, rimatr, n, dm, scale=1.0):
        r = np.asfortranarray(rimatr, dtype=np.float64)
        d = np.asfortranarray(dm, dtype=np.float64)
        out = np.empty(n * (n + 1) // 2)
        rc = self.L.cpu_vj_upper_with_rimatr(r.ctypes.data, n, r.shape[1], d.ctypes.data, scale, self.nthreads,
                                             out.ctypes.data)
        if rc:
            raise RuntimeError("cpu_vj failed")
        return out

    def vk_upper_with_ri_v(self, ri3fn, eigv, homo, occ, scale):
        r = np.asfortranarray(ri3fn, dtype=np.float64)
        n = r.shape[0]
        e = np.asfortranarray(eigv, dtype=np.float64)
        o = np.ascontiguousarray(occ, dtype=np.float64)
        out = np.empty(n * (n + 1) // 2)
        rc = self.L.cpu_vk_upper_with_ri_v(r.ctypes.data, n, r.shape[2], e.ctypes.data, e.shape[1], homo,
                                           o.ctypes.data, scale, self.nthreads, out.ctypes.data)
        if rc:
            raise RuntimeError("cpu_vk failed")
        return out
