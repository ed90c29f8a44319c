"""B200-native (sm_100a) RI Coulomb/exchange Fock build of REST (jeanwsr/rest).

The compute path is librest_b200.so (CUDA, C ABI in include/rest_b200.h);
this package is its host-side mirror of REST's vj/vk interface.
"""
from ._abi import RijkError, header_symbols, lib  # noqa: F401
from .rijk import RIJK, RIJKGroup, energy_contraction  # noqa: F401

__all__ = ["RIJK", "RijkError", "energy_contraction", "header_symbols", "lib"]
