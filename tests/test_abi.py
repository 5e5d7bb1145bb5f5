"""The C-ABI boundary without a GPU: the sm_100a library and the oracle load
and export exactly the entry points include/prism_b200.h declares."""
import ctypes
import os
import re

import pytest

from prism_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "prism_b200.h")).read()
    return sorted(set(re.findall(r"\b(prism_[a-z_]+)\s*\(", text)))


def test_header_matches_python_declarations():
    names = header_functions()
    assert sorted(_abi.exported_symbols("prism_")) == names


def test_library_exports_every_symbol():
    import prism_b200
    if not os.path.exists(prism_b200.LIB_PATH):
        pytest.skip("library not built")
    lib = ctypes.CDLL(prism_b200.LIB_PATH)
    for name in header_functions():
        assert hasattr(lib, name), name
    bound = prism_b200.lib()
    assert bound.last_error() is not None


def test_oracle_exports_every_symbol(orc):
    for name in header_functions():
        if name[len("prism_"):] in _abi.GPU_ONLY:
            continue  # device-side profiling has no CPU counterpart
        assert hasattr(orc.lib, "orc_" + name[len("prism_"):]), name


def test_status_strings(orc):
    orc.lib.orc_status_string.restype = ctypes.c_char_p
    assert orc.lib.orc_status_string(0) == b"OK"
    assert orc.lib.orc_status_string(7) == b"NO_BC_HANDLER"


@pytest.mark.parametrize("kind", ["hex", "tet"])
def test_mesh_host_build_and_index_checks(kind):
    # prism_mesh_create builds the PMesh on the host and checks that every index
    # (cells, faces, CSR and SELL-32 entries) fits 32 bits before it touches the
    # device: without a GPU the call gets exactly as far as creating the mesh's stream
    import prism_b200
    import torch
    from prism_b200 import api, io, meshgen
    if not os.path.exists(prism_b200.LIB_PATH):
        pytest.skip("library not built")
    unv = meshgen.box_hex(6, 5, 4, jitter=0.2, seed=1) if kind == "hex" else meshgen.box_tet(4, 3, 3)
    case = io.Case.from_dict(meshgen.PATCHES, {"T": {p: ("fixed", 0.0) for p in meshgen.PATCHES}}, {"T": {}})
    if torch.cuda.is_available():
        assert api.Mesh(unv, case, lib=prism_b200.lib()).n_cells > 0
        return
    with pytest.raises(_abi.PrismError) as err:
        api.Mesh(unv, case, lib=prism_b200.lib())
    assert err.value.status == _abi.CUDA_ERROR and "cudaStreamCreate" in str(err.value)
