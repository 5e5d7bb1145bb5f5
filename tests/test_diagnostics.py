"""Diagnostics (ops::div, ops::grad, the Courant number), cell-to-point
interpolation and VTU export, on the oracle.

The reference has no tests of its own for these (operations/operations.h,
monitor/courant.cpp, export.cpp), so the oracle is pinned on exact answers:
the divergence of a linear field from its exact face fluxes is its constant
divergence on any mesh with planar faces; the Courant number of a uniform flow
on a uniform grid is u dt / h; inverse-distance weights reproduce a constant
everywhere and a linear field at vertices equidistant from their cells. The
VTU files are read back and compared bit for bit with the arrays written."""
import os

import numpy as np
import pytest

from prism_b200 import PrismError, api, export, meshgen
from prism_b200 import _abi as A
from prism_b200.io import UnvData
from tests import cases

U0 = [1.0, 0.5, -0.25]


def box_mesh(lib, n=5, kind="hex", jitter=0.0, u_bc=("fixed", U0), empty_z=False, unv=None):
    if unv is None:
        gen = meshgen.box_hex if kind == "hex" else meshgen.box_tet
        unv = gen(n, n, n, jitter=jitter, seed=2)
    bcs = {p: u_bc for p in meshgen.PATCHES}
    tbc = {}
    if empty_z:
        bcs["back"] = bcs["front"] = ("empty", None)
        tbc = {"back": ("empty", None), "front": ("empty", None)}
    case = cases.box_case({"U": bcs, "T": tbc})
    return api.Mesh(unv, case, lib=lib)


def exact_fluxes(mesh, fn):
    """U(face centre) . S for a field given as fn(x, y, z) -> (3, n)."""
    ex = mesh.export()
    fc, nrm, area = ex["face_center"], ex["face_normal"], ex["face_area"]
    u = np.asarray(fn(fc[0], fc[1], fc[2]))
    return ((u[0] * nrm[0] + u[1] * nrm[1]) + u[2] * nrm[2]) * area


@pytest.mark.parametrize("kind, jitter", [("hex", 0.0), ("tet", 0.0), ("tet", 0.2)])
def test_div_uniform_field(orc, kind, jitter):
    # closed cells only: a non-planar (jittered hex) face's area * normal is not its
    # vector area (triangle-fan areas are summed, face.cpp:5-41), so sum(S) != 0 there
    mesh = box_mesh(orc, kind=kind, jitter=jitter)
    U = api.Vector("U", mesh, U0)
    d = api.ops.div(U)
    assert d.name == "div(U)"
    assert np.abs(d.values()).max() < 1e-12


@pytest.mark.parametrize("kind", ["hex", "tet"])
def test_div_linear_field_exact_fluxes(orc, kind):
    # planar faces: the face-centre flux of a linear field is exact, so is the divergence theorem
    mesh = box_mesh(orc, kind=kind, jitter=0.2 if kind == "tet" else 0.0)
    U = api.Vector("U", mesh, U0)
    U.set_face_flux(exact_fluxes(mesh, lambda x, y, z: (x + 2 * y, 2 * y - z, 3 * z + x)))
    np.testing.assert_allclose(api.ops.div(U).values(), 6.0, rtol=1e-12)


def test_courant_uniform_flow(orc):
    n, u, dt = 8, 2.0, 0.01
    mesh = box_mesh(orc, n=n, u_bc=("fixed", [u, 0.0, 0.0]))
    U = api.Vector("U", mesh, [u, 0.0, 0.0])
    co = api.monitor.courant_number(U, dt)
    assert co.name == "Co"
    np.testing.assert_allclose(co.values(), u * dt * n, rtol=1e-12)


def test_empty_faces_skipped(orc):
    # one cell layer: a z velocity crosses only the empty front/back faces, no flux is counted
    mesh = box_mesh(orc, u_bc=("fixed", [0.0, 0.0, 3.0]), empty_z=True, unv=meshgen.box_hex(6, 6, 1))
    U = api.Vector("U", mesh, [0.0, 0.0, 3.0])
    assert np.abs(api.monitor.courant_number(U, 1.0).values()).max() < 1e-12
    assert np.abs(api.ops.div(U).values()).max() < 1e-12
    f = U.face_flux()
    assert f.shape == (mesh.n_faces,)


def test_flux_field_with_face_fluxes(orc):
    # signed fluxes: a flux field from random face values obeys sum(div * V) = boundary flux
    mesh = box_mesh(orc, n=4, kind="tet", jitter=0.1)
    rng = np.random.default_rng(1)
    flux = rng.normal(size=mesh.n_faces)
    U = api.Vector("mdot", mesh, U0, bcs=mesh.case.bcs("U"))
    U.set_face_flux(flux)
    np.testing.assert_array_equal(U.face_flux(), flux)
    ex = mesh.export()
    vol = ex["cell_volume"]
    nb = mesh.info.n_boundary_faces
    total = (api.ops.div(U).values() * vol).sum()
    assert abs(total - flux[:nb].sum()) < 1e-11 * np.abs(flux).sum()
    co = api.monitor.courant_number(U, 0.5).values()
    cf_off, cf = ex["cell_face_offsets"], ex["cell_faces"]
    want = np.array([0.25 * np.abs(flux[cf[cf_off[c]:cf_off[c + 1]]]).sum() / vol[c]
                     for c in range(mesh.n_cells)])
    np.testing.assert_allclose(co, want, rtol=1e-14)


def test_topology(orc):
    n = 3
    mesh = box_mesh(orc, n=n)
    xyz, off, ids = mesh.topology()
    assert mesh.n_vertices == (n + 1) ** 3 == xyz.shape[0]
    assert np.all(np.diff(off) == 8) and off[-1] == ids.size
    unv = meshgen.box_hex(n, n, n)
    cells = [e for e in range(unv.n_elements) if unv.elem_kind[e] == A.ELEM_HEX]
    want = np.concatenate([unv.elem_nodes[unv.elem_offsets[e]:unv.elem_offsets[e + 1]] for e in cells])
    np.testing.assert_array_equal(ids, want)
    np.testing.assert_array_equal(xyz, unv.xyz)


@pytest.mark.parametrize("kind", ["hex", "tet"])
def test_cell_to_point_constant(orc, kind):
    mesh = box_mesh(orc, n=4, kind=kind, jitter=0.2)
    T = api.Scalar("T", mesh, 2.5)
    np.testing.assert_allclose(T.to_points(), 2.5, rtol=2e-15)  # a rounding per adjacent cell
    U = api.Vector("U", mesh, U0)
    np.testing.assert_allclose(U.to_points(), np.tile(U0, (mesh.n_vertices, 1)), rtol=2e-15)  # a rounding per adjacent cell


def test_cell_to_point_linear_interior_exact(orc):
    n = 6
    mesh = box_mesh(orc, n=n)
    cc = mesh.export()["cell_center"]
    xyz, _, _ = mesh.topology()
    T = api.Scalar("T", mesh, cc[0] + 2 * cc[1] + 3 * cc[2])
    pts = T.to_points()
    h = 1.0 / n
    inner = np.all((xyz > h / 2) & (xyz < 1 - h / 2), axis=1)
    assert inner.sum() == (n - 1) ** 3
    x = xyz[inner]
    np.testing.assert_allclose(pts[inner], x[:, 0] + 2 * x[:, 1] + 3 * x[:, 2], rtol=1e-13)


@pytest.mark.parametrize("ncomp", [1, 2, 3, 9])
def test_cell_to_point_components(orc, ncomp):
    # interleaved layout: component k of the result is the interpolation of component k
    mesh = box_mesh(orc, n=3, kind="tet", jitter=0.2)
    data = np.random.default_rng(ncomp).normal(size=(mesh.n_cells, ncomp))
    got = mesh.cell_to_point(data, ncomp).reshape(-1, ncomp)
    for k in range(ncomp):
        np.testing.assert_array_equal(got[:, k], mesh.cell_to_point(data[:, k].copy(), 1))


def test_vector_and_scalar_points_match_generic(orc):
    mesh = box_mesh(orc, n=3, jitter=0.2)
    rng = np.random.default_rng(3)
    U = api.Vector("U", mesh, rng.normal(size=(3, mesh.n_cells)))
    np.testing.assert_array_equal(U.to_points().reshape(-1), mesh.cell_to_point(U.values().T.copy(), 3))
    T = api.Scalar("T", mesh, rng.normal(size=mesh.n_cells))
    np.testing.assert_array_equal(T.to_points(), mesh.cell_to_point(T.values(), 1))


def test_vertex_without_cells_rejected(orc):
    unv = meshgen.box_hex(2, 2, 2)
    unv = UnvData(np.vstack([unv.xyz, [[5.0, 5.0, 5.0]]]), unv.elem_kind, unv.elem_offsets, unv.elem_nodes,
                  unv.groups)
    mesh = box_mesh(orc, unv=unv)
    T = api.Scalar("T", mesh, 1.0)
    with pytest.raises(PrismError) as e:
        T.to_points()
    assert e.value.status == A.INVALID_MESH and "Vertex 27" in str(e.value)


def test_ops_grad(orc):
    mesh = box_mesh(orc, n=4, jitter=0.2)
    cc = mesh.export()["cell_center"]
    T = api.Scalar("T", mesh, cc[0] * cc[1] + cc[2], bcs=mesh.case.bcs("T"))
    g = api.ops.grad(T)
    assert g.name == "grad(T)"
    np.testing.assert_array_equal(g.values(), T.grad())
    gy = api.ops.grad(T, 1)
    assert gy.name == "grad(T)_y"
    np.testing.assert_array_equal(gy.values(), T.grad()[1])
    U = api.Vector("U", mesh, np.stack([cc[0], 2 * cc[1], cc[0] + cc[2]]))
    t = api.ops.grad(U).values()
    comps = [U.x().grad(), U.y().grad(), U.z().grad()]
    for i in range(3):
        for j in range(3):
            np.testing.assert_array_equal(t[3 * i + j], comps[j][i])
    a = np.arange(9.0).reshape(3, 3)
    np.testing.assert_array_equal(api.ops.symm(a), 0.5 * (a + a.T))
    np.testing.assert_array_equal(api.ops.two_symm(a), a + a.T)
    assert abs(np.trace(api.ops.dev(a))) < 1e-15
    assert api.ops.double_contraction(a, np.eye(3)) == np.trace(a)


@pytest.mark.parametrize("mode", list(export.WriteMode))
def test_vtu_roundtrip(orc, tmp_path, mode):
    mesh = box_mesh(orc, n=3, kind="tet", jitter=0.2)
    rng = np.random.default_rng(7)
    T = api.Scalar("T", mesh, rng.normal(size=mesh.n_cells))
    U = api.Vector("U", mesh, rng.normal(size=(3, mesh.n_cells)))
    G = api.Tensor("G", mesh, rng.normal(size=(9, mesh.n_cells)))
    f = str(tmp_path / "out.vtu")
    export.to_vtu(f, [T], [U], [G], mode)
    r = export.read_vtu(f)
    xyz, off, ids = mesh.topology()
    np.testing.assert_array_equal(r["points"], xyz)
    np.testing.assert_array_equal(r["connectivity"], ids)
    np.testing.assert_array_equal(r["offsets"], off[1:])
    assert np.all(r["types"] == 10)
    assert list(r["cell_data"]) == ["T", "U", "G"] == list(r["point_data"])
    np.testing.assert_array_equal(r["cell_data"]["T"], T.values())
    np.testing.assert_array_equal(r["cell_data"]["U"], U.values().T)
    np.testing.assert_array_equal(r["cell_data"]["G"], G.values().T)
    np.testing.assert_array_equal(r["point_data"]["T"], T.to_points())
    np.testing.assert_array_equal(r["point_data"]["U"], U.to_points())
    np.testing.assert_array_equal(r["point_data"]["G"].reshape(-1),
                                  mesh.cell_to_point(G.values().T.copy(), 9))


def test_vtu_cell_types(orc, tmp_path):
    unv, case, _ = cases.load_golden("poisson_wedge")
    mesh = api.Mesh(unv, case, lib=orc)
    P = api.Scalar("P", mesh, 1.0)
    f = str(tmp_path / "w.vtu")
    export.to_vtu(f, scalars=[P])
    r = export.read_vtu(f)
    assert np.all(r["types"] == 13) and r["offsets"][-1] == 6 * mesh.n_cells
    mesh2 = box_mesh(orc, n=2)
    export.to_vtu(f, scalars=[api.Scalar("T", mesh2, 0.0)])
    assert np.all(export.read_vtu(f)["types"] == 12)


def test_vtu_errors(orc, tmp_path):
    m1, m2 = box_mesh(orc, n=2), box_mesh(orc, n=2)
    f = str(tmp_path / "x.vtu")
    export.to_vtu(f)
    assert not os.path.exists(f)  # no fields: nothing written
    with pytest.raises(PrismError) as e:
        export.to_vtu(f, [api.Scalar("T", m1, 0.0), api.Scalar("T", m2, 0.0)])
    assert e.value.status == A.INVALID_MESH
    with pytest.raises(ValueError):
        export.TimeWriter(str(tmp_path / "t"), 0)


def test_time_writer(orc, tmp_path):
    mesh = box_mesh(orc, n=2)
    T = api.Scalar("T", mesh, 1.0)
    prefix = str(tmp_path / "run")
    w = export.TimeWriter(prefix, write_interval=2)
    w.write_and_advance(0.1)  # nothing registered yet: no file
    w.add(T)
    for _ in range(4):
        w.write_and_advance(0.1)
    files = sorted(p.name for p in tmp_path.iterdir())
    assert files == ["run.pvd", "run_0002.vtu", "run_0004.vtu"]
    pvd = (tmp_path / "run.pvd").read_text()
    assert pvd.count("<DataSet") == 2
    assert f'timestep="0.2" file="{prefix}_0002.vtu"' in pvd
    assert f'timestep="0.4" file="{prefix}_0004.vtu"' in pvd
    reg = export.FieldRegistry()
    reg.add(T)
    reg.add(api.Vector("U", mesh, U0))
    reg.export_all(str(tmp_path / "all.vtu"), export.WriteMode.RawBinaryCompressed)
    assert list(export.read_vtu(str(tmp_path / "all.vtu"))["cell_data"]) == ["T", "U"]
