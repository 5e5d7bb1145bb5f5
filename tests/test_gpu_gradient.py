"""Cell gradients on the GPU vs the oracle: least squares and the level-scheduled
in-place Green-Gauss sweep reproduce the reference's cell-order sweep bit for bit
(including the sweep-to-sweep Gauss-Seidel seeding). Hex, tet and wedge cells
(6, 4 and 5 faces: one pass of the kernel's eight lanes per cell) on meshes of 10 to
59 dependency levels."""
import numpy as np
import pytest

from prism_b200 import _abi as A
from prism_b200 import api, meshgen
from tests import cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("grad", [A.GRAD_LEAST_SQUARES, A.GRAD_GREEN_GAUSS])
@pytest.mark.parametrize("kind", ["hex_small", "hex", "hex16", "tet", "wedge"])
def test_gradients_bit_exact(gpu, orc, grad, kind):
    if kind == "hex_small":
        unv, case = meshgen.box_hex(5, 4, 3, jitter=0.2, seed=10), cases.box_case({"T": {"left": ("fixed", 2.0)}})
    elif kind == "hex":
        unv, case = meshgen.box_hex(9, 7, 5, jitter=0.2, seed=11), cases.box_case({"T": {"left": ("fixed", 2.0)}})
    elif kind == "hex16":
        unv, case = meshgen.box_hex(16, 16, 16, jitter=0.2, seed=13), cases.box_case({"T": {"right": ("fixed", 1.0)}})
    elif kind == "tet":
        unv, case = meshgen.box_tet(4, 4, 4, jitter=0.2, seed=12), cases.box_case({"T": {"top": ("no-slip", 1.0)}})
    else:
        unv, case, _ = cases.load_golden("poisson_wedge")
    outs = []
    for lib in (gpu, orc):
        mesh = api.Mesh(unv, case, lib=lib)
        cc = mesh.export()["cell_center"]
        name = "T" if kind != "wedge" else "P"
        T = api.Scalar(name, mesh, np.sin(2 * cc[0]) * np.cos(cc[1]) + cc[2], grad_scheme=grad)
        sweeps = []
        for k in range(3):  # repeated sweeps: Green-Gauss seeds each sweep with the last one
            T.set_values(np.sin(2 * cc[0] + k) * np.cos(cc[1]) + cc[2])
            sweeps.append(T.grad())
        T.compute_all_cell_gradients()
        sweeps.append(T.grad())
        outs.append(np.array(sweeps))
    np.testing.assert_array_equal(outs[0], outs[1])


def test_face_values_and_fluxes(gpu, orc):
    unv = meshgen.box_hex(6, 5, 4, jitter=0.1, seed=3)
    case = cases.box_case({"T": {"left": ("fixed", 1.5), "bottom": ("symmetry", None)},
                           "U": {"left": ("fixed", [1.0, 0.0, 0.0]), "right": ("outlet", None),
                                 "bottom": ("symmetry", None), "top": ("no-slip", [0.0, 0.0, 0.0])}})
    outs = []
    for lib in (gpu, orc):
        mesh = api.Mesh(unv, case, lib=lib)
        cc = mesh.export()["cell_center"]
        T = api.Scalar("T", mesh, cc[0] + cc[1])
        U = api.Vector("U", mesh, np.stack([cc[0], cc[1] * cc[2], -cc[2]]))
        outs.append((T.face_values(), U.face_flux()))
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    np.testing.assert_array_equal(outs[0][1], outs[1][1])
