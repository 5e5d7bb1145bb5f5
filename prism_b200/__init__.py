"""prism_b200: B200 (sm_100a) implementation of Prism's finite-volume hot path.

The compute path is the in-tree CUDA library libprism_b200.so (C-ABI in
include/prism_b200.h). There is no CPU fallback: `lib()` raises if the library
is missing, and every call reports CUDA errors as a PrismError.
"""
import ctypes
import os

from . import _abi
from ._abi import PrismError  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libprism_b200.so")
_bound = None


def lib():
    """The bound sm_100a library (loaded once)."""
    global _bound
    if _bound is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run `python -m prism_b200.build`")
        _bound = _abi.bind(ctypes.CDLL(LIB_PATH), "prism_")
    return _bound
