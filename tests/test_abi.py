"""CPU checks of the C ABI library: it builds, loads, exports every symbol the
public header declares, and refuses to run without an sm_100 GPU (no fallback)."""
import ctypes as C

import pytest

from rest_b200 import _abi, build


@pytest.fixture(scope="module")
def L():
    build.build()
    return C.CDLL(str(_abi.LIB_PATH))


def test_every_declared_symbol_is_exported(L):
    names = _abi.header_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_binding_signatures_cover_the_header():
    assert set(_abi.header_symbols()) <= set(_abi.SIGNATURES)


def test_status_strings(L):
    L.rijk_status_string.restype = C.c_char_p
    assert L.rijk_status_string(0) == b"ok"
    assert b"positive definite" in L.rijk_status_string(3)


def test_energy_contraction_runs_on_host(L):
    import numpy as np

    from oracle import rijk_oracle as O
    from rest_b200 import energy_contraction

    rng = np.random.default_rng(3)
    a = rng.standard_normal(28)
    b = rng.standard_normal(28)
    assert abs(energy_contraction(a, b) - O.par_energy_contraction(a, b)) < 1e-13


def test_context_creation_fails_loudly_without_a_gpu(L):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    from rest_b200 import RIJK, RijkError

    with pytest.raises(RijkError):
        RIJK(0)
