"""CPU oracle of the Prism hot path -- TEST INFRASTRUCTURE, not product code.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this
package, and only to check the GPU results against (or, for the timed CPU
baseline, as the restated reference implementation). It exposes the same C-ABI as the sm_100a
library with the prefix ``orc_``.
"""
import ctypes
import os
import sys

_HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(_HERE)) if os.path.dirname(_HERE) not in sys.path else None

from prism_b200 import _abi  # noqa: E402  (struct layouts of the shared C-ABI)

from . import build as _build  # noqa: E402

_bound = None


def lib():
    """Bound oracle entry points (built on first use when the source is newer)."""
    global _bound
    if _bound is None:
        path = _build.LIB
        if os.path.exists(_build.SRC):
            path = _build.build()
        _bound = _abi.bind(ctypes.CDLL(path), "orc_")
    return _bound
