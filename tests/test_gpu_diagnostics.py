"""Diagnostics and point data on the GPU vs the oracle, bit for bit.

ops::div, the Courant number and cellToPoint are gathers with the
reference's operation order (compiled without FMA contraction): on the same
inputs the device results equal the oracle's exactly, on hexahedra, wedges
and tetrahedra, with boundary-condition fluxes, stored face fluxes and empty
patches. At 128^3 cells the size-independent properties are checked."""
import numpy as np
import pytest

from prism_b200 import api, export, meshgen
from tests import cases
from tests.test_diagnostics import box_mesh

pytestmark = pytest.mark.gpu


def _meshes(lib):
    unv, case, _ = cases.load_golden("poisson_wedge")
    return {
        "hex-jitter": box_mesh(lib, n=7, jitter=0.25),
        "tet": box_mesh(lib, n=5, kind="tet", jitter=0.2),
        "cavity-empty": box_mesh(lib, empty_z=True, unv=meshgen.box_hex(9, 9, 1)),
        "wedge": api.Mesh(unv, case, lib=lib),
    }


def _fields(mesh, seed):
    rng = np.random.default_rng(seed)
    n = mesh.n_cells
    bcs = mesh.case.bcs("U") if "U" in mesh.case.fields else None
    U = api.Vector("U", mesh, rng.normal(size=(3, n)), bcs=bcs if bcs is not None else api._default_bcs(mesh))
    T = api.Scalar("T", mesh, rng.normal(size=n), bcs=api._default_bcs(mesh))
    return U, T, rng


@pytest.mark.parametrize("name", ["hex-jitter", "tet", "cavity-empty", "wedge"])
def test_diagnostics_bitexact(gpu, orc, name):
    out = {}
    for which, lib in (("gpu", gpu), ("orc", orc)):
        mesh = _meshes(lib)[name]
        U, T, rng = _fields(mesh, 11)
        r = {}
        if "U" in mesh.case.fields:  # fluxes through the boundary handlers
            r["div_bc"] = api.ops.div(U).values()
            r["co_bc"] = api.monitor.courant_number(U, 0.37).values()
        U.set_face_flux(rng.normal(size=mesh.n_faces))
        r["div_ff"] = api.ops.div(U).values()
        r["co_ff"] = api.monitor.courant_number(U, 0.37).values()
        r["pts_T"] = T.to_points()
        r["pts_U"] = U.to_points()
        for nc in (2, 9):
            r[f"pts_{nc}"] = mesh.cell_to_point(rng.normal(size=(mesh.n_cells, nc)), nc)
        r["topology"] = np.concatenate([a.reshape(-1).astype(np.float64) for a in mesh.topology()])
        out[which] = r
    for k in out["orc"]:
        np.testing.assert_array_equal(out["gpu"][k], out["orc"][k], err_msg=f"{name}:{k}")


def test_export_files_match(gpu, orc, tmp_path):
    got = {}
    for which, lib in (("gpu", gpu), ("orc", orc)):
        mesh = box_mesh(lib, n=4, kind="tet", jitter=0.2)
        U, T, rng = _fields(mesh, 5)
        G = api.Tensor("G", mesh, rng.normal(size=(9, mesh.n_cells)))
        f = str(tmp_path / f"{which}.vtu")
        export.to_vtu(f, [T, api.ops.div(U)], [U], [G], export.WriteMode.RawBinaryCompressed)
        got[which] = open(f, "rb").read()
    assert got["gpu"] == got["orc"]


def test_large_mesh_properties(gpu):
    n = 128
    mesh = box_mesh(gpu, n=n, u_bc=("fixed", [2.0, 0.0, 0.0]))
    U = api.Vector("U", mesh, [2.0, 0.0, 0.0])
    np.testing.assert_allclose(api.monitor.courant_number(U, 1e-3).values(), 2.0 * 1e-3 * n, rtol=1e-12)
    assert np.abs(api.ops.div(U).values()).max() < 1e-9
    T = api.Scalar("T", mesh, 1.5, bcs=api._default_bcs(mesh))
    pts = T.to_points()
    assert pts.shape == ((n + 1) ** 3,)
    np.testing.assert_allclose(pts, 1.5, rtol=2e-15)
    cc = mesh.export()["cell_center"]
    T.set_values(cc[0] - cc[1] + 0.5 * cc[2])
    xyz = mesh.topology()[0]
    h = 1.0 / n
    inner = np.all((xyz > h / 2) & (xyz < 1 - h / 2), axis=1)
    x = xyz[inner]
    np.testing.assert_allclose(T.to_points()[inner], x[:, 0] - x[:, 1] + 0.5 * x[:, 2], rtol=1e-12, atol=1e-14)


def _bcs(mesh, vector=False):
    """Boundary conditions on every non-empty patch, alternating kinds: a fixed value
    (a vector for U) and zero gradient."""
    arr = (api.A.BC * max(1, mesh.info.n_patches))()
    for q in range(mesh.info.n_patches):
        if mesh.case.patch_is_empty[q]:
            arr[q].kind = api.A.BC_EMPTY
        elif q % 2 == 0:
            arr[q].kind = api.A.BC_FIXED
            if vector:
                arr[q].value_kind = api.A.BCV_VECTOR
                arr[q].vector[:] = [0.2 * q, -0.1, 0.05 * q]
            else:
                arr[q].value_kind = api.A.BCV_SCALAR
                arr[q].value = 0.3 + 0.1 * q
        else:
            arr[q].kind = api.A.BC_ZERO_GRADIENT
    return arr


@pytest.mark.parametrize("name", ["hex-jitter", "tet", "cavity-empty", "wedge"])
def test_rhie_chow_and_grad_scheme_bitexact(gpu, orc, name):
    """ops::rhieChowCorrectFace over the faces (prism_rhie_chow) with a full random
    tensor D, and Scalar::setGradScheme switching p's gradient scheme between calls:
    face velocities, fluxes and gradients equal the oracle's bit for bit."""
    out = {}
    for which, lib in (("gpu", gpu), ("orc", orc)):
        mesh = _meshes(lib)[name]
        rng = np.random.default_rng(23)
        n = mesh.n_cells
        U = api.Vector("U", mesh, rng.normal(size=(3, n)), bcs=_bcs(mesh, vector=True))
        p = api.Scalar("p", mesh, rng.normal(size=n), bcs=_bcs(mesh))
        a = rng.normal(size=(3, 3, n))
        d = np.einsum("ikc,jkc->ijc", a, a) + 0.5 * np.eye(3)[:, :, None]  # symmetric positive definite per cell
        D = api.Tensor("D", mesh, d.reshape(9, n))
        mdot = U.clone()
        r = {}
        for k, scheme in enumerate((api.A.GRAD_LEAST_SQUARES, api.A.GRAD_GREEN_GAUSS, api.A.GRAD_LEAST_SQUARES)):
            p.set_grad_scheme(scheme)
            api.ops.rhie_chow(mdot, U, D, p)
            r[f"flux_{k}"] = mdot.face_flux()
            r[f"grad_{k}"] = p.grad()
            p.set_values(p.values() * 1.5 + 0.25)
        out[which] = r
    for k in out["orc"]:
        np.testing.assert_array_equal(out["gpu"][k], out["orc"][k], err_msg=f"{name}:{k}")
