"""Structural invariants of the UNV -> PMesh conversion, the checks of the
reference's tests/test_unv_converter.cpp:10-72 (whose cylinder mesh is missing
from the reference checkout) applied to every reference mesh that is present
and to synthetic boxes of known volume and surface area:
  * every interior face's normal points from its owner to its neighbour;
  * every face of a non-empty boundary patch has its normal pointing out of its
    owner (the reference uses a boundary face's area vector as the owner's
    outward vector, mesh/utilities.cpp:15-18); faces of empty patches (the
    front and back of the 2-D meshes) may point either way, as the UNV node order
    gives them, since nothing reads them;
  * boundary faces have no neighbour, interior faces have one;
  * the cell volumes add up to the domain volume (the boundary integral
    (1/3) sum(x_f . S_f) for the reference meshes, the box volume for the boxes),
    and the boundary face areas to the box's surface area.
Checked on the oracle's conversion; the GPU path's conversion is bit-exact
against it (tests/test_gpu_mesh.py)."""
import numpy as np
import pytest

from prism_b200 import api, io, meshgen
from tests import cases

GOLDEN = ["poisson_hex", "poisson_wedge", "versteeg_advection_1d", "versteeg_trans_1d", "coarse_pipe",
          "cavity_hex", "duct_simple"]


def _check_orientation(e, nb, empty_patch):
    """Returns the sign that turns each boundary face's area vector outward."""
    own, nbr = e["owner"], e["neighbor"]
    n, fc, cc = e["face_normal"], e["face_center"], e["cell_center"]
    assert np.all(nbr[:nb] < 0) and np.all(nbr[nb:] >= 0)
    d = cc[:, nbr[nb:]] - cc[:, own[nb:]]
    assert np.all(np.einsum("ij,ij->j", n[:, nb:], d) > 0), "interior normal pointing from neighbour to owner"
    out = np.einsum("ij,ij->j", n[:, :nb], fc[:, :nb] - cc[:, own[:nb]])
    empty = np.asarray(empty_patch, bool)[e["face_patch"][:nb]]
    assert np.all(out[~empty] > 0), "boundary normal pointing into the domain"
    return np.sign(out)


@pytest.mark.parametrize("name", GOLDEN)
def test_reference_meshes(orc, name):
    unv, case, _ = cases.load_golden(name)
    mesh = api.Mesh(unv, case, lib=orc)
    e, nb = mesh.export(), mesh.info.n_boundary_faces
    sign = _check_orientation(e, nb, case.patch_is_empty)
    S = e["face_normal"][:, :nb] * (sign * e["face_area"][:nb])
    boundary_volume = np.einsum("ij,ij->", e["face_center"][:, :nb], S) / 3.0
    vol = e["cell_volume"].sum()
    print(f"{name}: {mesh.n_cells} cells, volume {vol:.10g}, boundary integral {boundary_volume:.10g}")
    assert np.all(e["cell_volume"] > 0)
    assert abs(vol - boundary_volume) <= 1e-9 * abs(vol)


@pytest.mark.parametrize("kind", ["hex", "tet"])
def test_box_volume_and_area(orc, kind):
    L = (1.5, 2.0, 0.5)
    gen = meshgen.box_hex if kind == "hex" else meshgen.box_tet
    unv = gen(5, 4, 3, lengths=L, origin=(-0.25, 1.0, 3.0))
    case = io.Case.from_dict(meshgen.PATCHES, {"T": {p: ("fixed", 0.0) for p in meshgen.PATCHES}}, {"T": {}})
    mesh = api.Mesh(unv, case, lib=orc)
    e, nb = mesh.export(), mesh.info.n_boundary_faces
    _check_orientation(e, nb, case.patch_is_empty)
    assert abs(e["cell_volume"].sum() - L[0] * L[1] * L[2]) < 1e-12
    area = 2 * (L[0] * L[1] + L[1] * L[2] + L[0] * L[2])
    assert abs(e["face_area"][:nb].sum() - area) < 1e-12
