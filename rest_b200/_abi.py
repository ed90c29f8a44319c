"""ctypes binding of librest_b200.so (declarations in include/rest_b200.h).

The library is loaded from this package directory only.  There is no CPU
fallback: if the shared library is missing the import of any wrapper fails
with an error telling how to build it, and ``RIJK`` contexts fail to open
without an sm_100 GPU.
"""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "librest_b200.so"
HEADER_PATH = Path(__file__).resolve().parent.parent / "include" / "rest_b200.h"

STATUS = {
    0: "RIJK_OK",
    1: "RIJK_ERR_ARG",
    2: "RIJK_ERR_CUDA",
    3: "RIJK_ERR_NOT_SPD",
    4: "RIJK_ERR_NO_TENSOR",
    5: "RIJK_ERR_TIMEOUT",
    6: "RIJK_ERR_NOMEM",
    7: "RIJK_ERR_NONFINITE",
    8: "RIJK_ERR_TOO_LARGE",
}


class RijkError(RuntimeError):
    def __init__(self, status: int, message: str, failed_pivot: int = 0):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status
        self.failed_pivot = failed_pivot


_lib = None


class RijkShells(C.Structure):
    """struct rijk_shells of include/rest_b200.h."""

    _fields_ = [
        ("nshell", C.c_int64),
        ("l", C.POINTER(C.c_int32)),
        ("nprim", C.POINTER(C.c_int32)),
        ("prim_off", C.POINTER(C.c_int64)),
        ("exps", C.POINTER(C.c_double)),
        ("coefs", C.POINTER(C.c_double)),
        ("centers", C.POINTER(C.c_double)),
    ]


_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)
_ctxp = C.c_void_p

# name -> (restype, argtypes)
SIGNATURES = {
    "rijk_ctx_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "rijk_ctx_destroy": (C.c_int, [_ctxp]),
    "rijk_ctx_last_error": (C.c_char_p, [_ctxp]),
    "rijk_status_string": (C.c_char_p, [C.c_int]),
    "rijk_ctx_info": (C.c_int, [_ctxp, _i64p, _i64p, _i64p]),
    "rijk_ctx_stream": (C.c_void_p, [_ctxp]),
    "rijk_ctx_tensor": (C.c_int, [_ctxp, C.POINTER(C.c_void_p), _i64p]),
    "rijk_ctx_synchronize": (C.c_int, [_ctxp, C.c_void_p]),
    "rijk_kernel_launches": (C.c_int64, []),
    "rijk_ctx_profile": (C.c_int, [_ctxp, C.c_int]),
    "rijk_ctx_set_tiles": (C.c_int, [_ctxp, C.c_int, C.c_int]),
    "rijk_ctx_get_tiles": (C.c_int, [_ctxp, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "rijk_ctx_pin_buffers": (C.c_int, [_ctxp, C.c_int]),
    "rijk_ctx_set_wait_budget": (C.c_int, [_ctxp, C.c_int64]),
    "rijk_group_create": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "rijk_group_destroy": (C.c_int, [C.c_void_p]),
    "rijk_group_jk_occ_dev": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_double,
                                        C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p]),
    "rijk_group_synchronize": (C.c_int, [C.c_void_p, C.c_void_p]),
    "rijk_diis_coefficients_dev": (
        C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p],
    ),
    "rijk_eigh_batched_dev": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_double, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "rijk_ctx_selftest_timeout": (C.c_int, [_ctxp]),
    "rijk_ctx_autotune": (
        C.c_int,
        [_ctxp, C.c_int64, C.c_int64, C.POINTER(C.c_int), C.POINTER(C.c_int), _dp],
    ),
    "rijk_ctx_profile_read": (C.c_int, [_ctxp, _dp, _i64p]),
    "rijk_set_rimatr": (C.c_int, [_ctxp, C.c_void_p, C.c_int64, C.c_int64]),
    "rijk_set_ri3fn": (C.c_int, [_ctxp, C.c_void_p, C.c_int64, C.c_int64]),
    "rijk_get_rimatr": (C.c_int, [_ctxp, C.c_void_p]),
    "rijk_tensor_alloc": (C.c_int, [_ctxp, C.c_int64, C.c_int64]),
    "rijk_tensor_load_rows_dev": (C.c_int, [_ctxp, C.c_void_p, C.c_int64, C.c_int64, C.c_int, C.c_void_p]),
    "rijk_build_rimatr_cholesky": (C.c_int, [_ctxp, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, _i64p]),
    "rijk_fit_rimatr": (C.c_int, [_ctxp, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64]),
    "rijk_vj_upper_with_ri_v": (C.c_int, [_ctxp, C.c_void_p, C.c_int, C.c_double, C.c_void_p]),
    "rijk_vj_upper_with_rimatr_v": (C.c_int, [_ctxp, C.c_void_p, C.c_int, C.c_double, C.c_void_p]),
    "rijk_vj_full_with_ri_v": (C.c_int, [_ctxp, C.c_void_p, C.c_int, C.c_double, C.c_void_p]),
    "rijk_vk_upper_with_ri_v": (
        C.c_int,
        [_ctxp, C.c_void_p, C.c_int64, _i64p, C.c_void_p, C.c_int, C.c_double, C.c_void_p],
    ),
    "rijk_vk_upper_with_ri_v_use_dm_only": (C.c_int, [_ctxp, C.c_void_p, C.c_int, C.c_double, C.c_void_p]),
    "rijk_vk_upper_with_rimatr_use_dm_only": (C.c_int, [_ctxp, C.c_void_p, C.c_int, C.c_double, C.c_void_p]),
    "rijk_vk_full_fromdm_with_ri_v": (C.c_int, [_ctxp, C.c_void_p, C.c_int, C.c_double, C.c_void_p]),
    "rijk_vj_upper_dev": (C.c_int, [_ctxp, C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_void_p, C.c_void_p]),
    "rijk_vk_upper_occ_dev": (
        C.c_int,
        [_ctxp, C.c_void_p, C.c_int64, _i64p, C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_void_p],
    ),
    "rijk_vk_upper_dm_dev": (C.c_int, [_ctxp, C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_void_p]),
    "rijk_vjk_upper_with_ri_v": (
        C.c_int,
        [_ctxp, C.c_void_p, C.c_int64, _i64p, C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_void_p],
    ),
    "rijk_vjk_upper_occ_dev": (
        C.c_int,
        [_ctxp, C.c_void_p, C.c_int64, _i64p, C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_void_p,
         C.c_void_p],
    ),
    "rijk_vk_upper_occ_split_dev": (
        C.c_int,
        [_ctxp, C.c_void_p, C.c_int64, _i64p, C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_void_p],
    ),
    "rijk_vjk_upper_lowrank_split_dev": (
        C.c_int,
        [_ctxp, C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_int, C.c_void_p,
         C.c_void_p, C.c_void_p],
    ),
    "rijk_vk_upper_lowrank_split_dev": (
        C.c_int,
        [_ctxp, C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_int, C.c_void_p, C.c_void_p],
    ),
    "rijk_vj_upper_noalloc": (
        C.c_int,
        [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_void_p,
         C.c_void_p],
    ),
    "rijk_density_matrix": (
        C.c_int,
        [_ctxp, C.c_void_p, C.c_int64, C.c_int64, _i64p, C.c_void_p, C.c_int, C.c_void_p],
    ),
    "rijk_energy_contraction": (C.c_double, [C.c_void_p, C.c_void_p, C.c_int64]),
    "rijk_ao2mo": (
        C.c_int,
        [_ctxp, C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int, C.c_void_p],
    ),
    "rijk_int1e": (C.c_int, [C.POINTER(RijkShells), C.c_void_p, C.c_int, C.c_int, _dp, _dp, _dp]),
    "rijk_int2c2e": (C.c_int, [C.POINTER(RijkShells), C.c_void_p, _dp]),
    "rijk_int3c2e": (C.c_int, [C.POINTER(RijkShells), C.POINTER(RijkShells), C.c_void_p, _dp]),
    "rijk_int2c2e_dev": (C.c_int, [C.POINTER(RijkShells), C.c_void_p, C.c_void_p, C.c_void_p]),
    "rijk_int3c2e_dev": (
        C.c_int,
        [C.POINTER(RijkShells), C.POINTER(RijkShells), C.c_void_p, C.c_void_p, C.c_void_p],
    ),
    "rijk_build_rimatr_from_shells": (
        C.c_int,
        [_ctxp, C.POINTER(RijkShells), C.POINTER(RijkShells), C.c_void_p, C.c_void_p, _i64p],
    ),
    "rijk_mlp_linear_fwd": (
        C.c_int,
        [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int, C.c_void_p, C.c_void_p,
         C.c_void_p, C.c_void_p],
    ),
    "rijk_mlp_linear_bwd": (
        C.c_int,
        [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int, C.c_void_p,
         C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    ),
    "rijk_mlp_masked_mse": (
        C.c_int,
        [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p],
    ),
    "rijk_mlp_adam": (
        C.c_int,
        [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_double, C.c_double,
         C.c_double, C.c_double, C.c_int64, C.c_void_p],
    ),
    "rijk_mlp_to_bf16": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]),
    "rijk_guess_assemble": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                      C.c_void_p]),
    "rijk_guess_geometry": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "rijk_guess_pairs": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p]),
}


def header_symbols() -> list[str]:
    """Every function declared in include/rest_b200.h."""
    txt = HEADER_PATH.read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(rijk_[a-z0-9_]+)\s*\(", txt)))


def lib() -> C.CDLL:
    """Load (once) the in-tree shared library; raise if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m rest_b200.build` "
            "(there is no CPU fallback for the RI J/K build)"
        )
    L = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L
