"""Mesh flattening on the GPU path vs the oracle: face order, owners, neighbours,
patches, cell face lists and the device-built CSR pattern bit for bit, geometry
bit for bit (same host arithmetic)."""
import numpy as np
import pytest

from prism_b200 import api, meshgen
from tests import cases

pytestmark = pytest.mark.gpu

INT_KEYS = ["owner", "neighbor", "face_patch", "cell_face_offsets", "cell_faces", "csr_rowptr", "csr_col",
            "patch_face_offsets", "patch_faces"]
FLOAT_KEYS = ["face_area", "face_normal", "face_center", "cell_volume", "cell_center"]


def _meshes():
    yield "poisson_hex", *cases.load_golden("poisson_hex")[:2]
    yield "poisson_wedge", *cases.load_golden("poisson_wedge")[:2]
    yield "duct_simple", *cases.load_golden("duct_simple")[:2]
    case = cases.box_case({"T": {}})
    yield "hex_jitter", meshgen.box_hex(7, 5, 6, jitter=0.2, seed=1), case
    yield "tets", meshgen.box_tet(4, 5, 3, jitter=0.15, seed=2), case


@pytest.mark.parametrize("name, unv, case", list(_meshes()), ids=lambda v: v if isinstance(v, str) else "")
def test_mesh_bit_exact(gpu, orc, name, unv, case):
    g = api.Mesh(unv, case, lib=gpu)
    o = api.Mesh(unv, case, lib=orc)
    for attr in ("n_cells", "n_faces", "n_boundary_faces", "n_nonempty_boundary_faces", "nnz", "n_gs_levels"):
        assert getattr(g.info, attr) == getattr(o.info, attr), attr
    eg, eo = g.export(), o.export()
    for k in INT_KEYS:
        np.testing.assert_array_equal(eg[k], eo[k], err_msg=k)
    for k in FLOAT_KEYS:
        np.testing.assert_array_equal(eg[k], eo[k], err_msg=k)
