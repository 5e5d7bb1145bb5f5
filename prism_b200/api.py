"""Python mirror of Prism's operator API over the C-ABI.

Class and argument names follow the reference (field::Scalar/Vector/Tensor,
eqn::Transport, scheme::convection::*, scheme::diffusion::*, scheme::source::*,
solver::BiCGSTAB/Jacobi, algo::IncompressibleSIMPLE/PRIME/PISO); errors are
raised as `PrismError` where the reference throws. Every object drives one
loaded C-ABI library: by default the sm_100a library (`prism_b200.lib()`).
The `lib` argument of `Mesh` lets a test build the same case on another
library exposing the same ABI (the CPU oracle) to compare the two.
"""
import ctypes as C
from dataclasses import dataclass, fields as dc_fields
from typing import Optional

import numpy as np

from . import _abi as A
from .io import Case, UnvData


def _f64p(a):
    return a.ctypes.data_as(A.pf64) if a is not None else None


def _default_lib():
    from . import lib
    return lib()


class Mesh:
    """PMesh built from a UNV-form mesh and the case's patches (UnvToPMeshConverter)."""

    def __init__(self, unv: UnvData, case: Case, lib=None):
        self.lib = lib if lib is not None else _default_lib()
        self.case = case
        self._keep = []
        d = A.UnvMesh()
        d.n_nodes = unv.n_nodes
        d.xyz = _f64p(unv.xyz)
        d.n_elements = unv.n_elements
        d.elem_kind = unv.elem_kind.ctypes.data_as(A.pi32)
        d.elem_offsets = unv.elem_offsets.ctypes.data_as(A.pi64)
        d.elem_nodes = unv.elem_nodes.ctypes.data_as(A.pi64)
        gnames = (C.c_char_p * max(1, len(unv.groups)))(*[g[0].encode() for g in unv.groups])
        gvert = np.array([1 if g[1] else 0 for g in unv.groups] or [0], dtype=np.int32)
        goff = np.zeros(len(unv.groups) + 1, dtype=np.int64)
        for i, g in enumerate(unv.groups):
            goff[i + 1] = goff[i] + len(g[2])
        gel = (np.concatenate([g[2] for g in unv.groups]).astype(np.int64)
               if unv.groups else np.zeros(1, np.int64))
        d.n_groups = len(unv.groups)
        d.group_names = gnames
        d.group_is_vertex = gvert.ctypes.data_as(A.pi32)
        d.group_offsets = goff.ctypes.data_as(A.pi64)
        d.group_elements = gel.ctypes.data_as(A.pi64)
        pnames = (C.c_char_p * max(1, len(case.patch_names)))(*[p.encode() for p in case.patch_names])
        pempty = np.array([1 if e else 0 for e in case.patch_is_empty] or [0], dtype=np.int32)
        d.n_patches = len(case.patch_names)
        d.patch_names = pnames
        d.patch_is_empty = pempty.ctypes.data_as(A.pi32)
        h = C.c_void_p()
        self.lib.check(self.lib.mesh_from_unv(C.byref(d), C.byref(h)))
        self.h = h
        info = A.MeshInfo()
        self.lib.check(self.lib.mesh_info(self.h, C.byref(info)))
        self.info = info
        self.n_cells = info.n_cells
        self.n_faces = info.n_faces
        self.n_vertices = info.n_vertices

    def export(self):
        """Flattened PMesh + CSR pattern as numpy arrays (SoA vectors)."""
        i, nc, nf = self.info, self.info.n_cells, self.info.n_faces
        cfo = np.zeros(nc + 1, np.int64)
        e = A.MeshExport()
        e.cell_face_offsets = cfo.ctypes.data_as(A.pi64)
        self.lib.check(self.lib.mesh_export(self.h, C.byref(e)))
        pfo = np.zeros(i.n_patches + 1, np.int64)
        e = A.MeshExport()
        e.patch_face_offsets = pfo.ctypes.data_as(A.pi64)
        self.lib.check(self.lib.mesh_export(self.h, C.byref(e)))
        out = dict(
            owner=np.zeros(nf, np.int64), neighbor=np.zeros(nf, np.int64),
            face_patch=np.zeros(nf, np.int32), face_area=np.zeros(nf), face_normal=np.zeros(3 * nf),
            face_center=np.zeros(3 * nf), cell_volume=np.zeros(nc), cell_center=np.zeros(3 * nc),
            cell_face_offsets=cfo, cell_faces=np.zeros(max(1, cfo[-1]), np.int64),
            csr_rowptr=np.zeros(nc + 1, np.int64), csr_col=np.zeros(max(1, i.nnz), np.int64),
            patch_face_offsets=pfo, patch_faces=np.zeros(max(1, pfo[-1]), np.int64),
            vertex_coords=np.zeros(3 * i.n_vertices), cell_vertex_offsets=np.zeros(nc + 1, np.int64),
            cell_vertices=np.zeros(max(1, i.n_cell_vertices), np.int64),
            cell_original=np.zeros(nc, np.int64))
        e = A.MeshExport()
        for k, v in out.items():
            ptype = dict(e._fields_)[k]
            setattr(e, k, v.ctypes.data_as(ptype))
        self.lib.check(self.lib.mesh_export(self.h, C.byref(e)))
        for k in ("face_normal", "face_center"):
            out[k] = out[k].reshape(3, nf)
        out["cell_center"] = out["cell_center"].reshape(3, nc)
        out["vertex_coords"] = out["vertex_coords"].reshape(3, i.n_vertices)
        return out

    def reorder(self, reverse=False):
        """CuthillMckee(mesh).reorder(reverse) (mesh/reorder.cpp): renumbers the cells in
        (reverse) Cuthill-McKee order. Call before creating fields on the mesh;
        export()["cell_original"] maps each new cell id to its id before reordering."""
        self.lib.check(self.lib.mesh_reorder(self.h, 1 if reverse else 0))
        self._topology = None

    def topology(self):
        """Vertices (n_vertices, 3) and the cells' vertex lists (offsets n_cells+1,
        vertex ids in UNV element node order)."""
        if getattr(self, "_topology", None) is None:
            i = self.info
            xyz = np.zeros(3 * i.n_vertices)
            off = np.zeros(i.n_cells + 1, np.int64)
            ids = np.zeros(max(1, i.n_cell_vertices), np.int64)
            e = A.MeshExport()
            e.vertex_coords = xyz.ctypes.data_as(A.pf64)
            e.cell_vertex_offsets = off.ctypes.data_as(A.pi64)
            e.cell_vertices = ids.ctypes.data_as(A.pi64)
            self.lib.check(self.lib.mesh_export(self.h, C.byref(e)))
            self._topology = (xyz.reshape(3, -1).T.copy(), off, ids[:i.n_cell_vertices])
        return self._topology

    def cell_to_point(self, cell_data, n_components=1):
        """cellToPoint (export.cpp:73-111): inverse-distance weighted vertex values
        of interleaved cell data (n_cells * n_components), interleaved per vertex."""
        d = np.ascontiguousarray(cell_data, dtype=np.float64).reshape(-1)
        if d.size != self.n_cells * n_components:
            raise ValueError("cell_data must hold n_cells * n_components values")
        out = np.zeros(self.n_vertices * n_components)
        self.lib.check(self.lib.cell_to_point(self.h, _f64p(d), int(n_components), _f64p(out)))
        return out

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.mesh_destroy(self.h)
            self.h = None


class Scalar:
    """field::Scalar. BCs and gradient scheme come from the case unless given."""

    def __init__(self, name, mesh: Mesh, value=0.0, grad_scheme=None, bcs=None, _handle=None,
                 _owner=None):
        self.mesh, self.lib, self.name = mesh, mesh.lib, name
        self._owner = _owner
        if _handle is not None:
            self.h = _handle
            self._borrowed = True
            return
        self._borrowed = False
        vals = np.full(mesh.n_cells, float(value)) if np.isscalar(value) else \
            np.ascontiguousarray(value, dtype=np.float64)
        gs = mesh.case.grad_scheme(name) if grad_scheme is None else grad_scheme
        if bcs is None:
            bcs = mesh.case.bcs(name) if name in mesh.case.fields else _default_bcs(mesh)
        self._bcs = bcs
        h = C.c_void_p()
        self.lib.check(self.lib.scalar_create(mesh.h, name.encode(), _f64p(vals), gs, bcs, C.byref(h)))
        self.h = h

    def values(self):
        out = np.zeros(self.mesh.n_cells)
        self.lib.check(self.lib.scalar_get_values(self.h, _f64p(out)))
        return out

    def set_values(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        self.lib.check(self.lib.scalar_set_values(self.h, _f64p(v)))

    def set_face_values(self, fv):
        fv = None if fv is None else np.ascontiguousarray(fv, dtype=np.float64)
        self.lib.check(self.lib.scalar_set_face_values(self.h, _f64p(fv)))

    def clear_face_values(self):
        self.set_face_values(None)

    def face_values(self):
        out = np.zeros(self.mesh.n_faces)
        self.lib.check(self.lib.scalar_face_values(self.h, _f64p(out)))
        return out

    def grad(self):
        """gradAtCell for every cell, shape (3, n_cells)."""
        out = np.zeros(3 * self.mesh.n_cells)
        self.lib.check(self.lib.scalar_grad(self.h, _f64p(out)))
        return out.reshape(3, -1)

    def compute_all_cell_gradients(self):
        self.lib.check(self.lib.scalar_compute_gradients(self.h))

    def set_grad_scheme(self, grad_scheme):
        """Scalar::setGradScheme (scalar.cpp:252-258): A.GRAD_LEAST_SQUARES or
        A.GRAD_GREEN_GAUSS; the new scheme starts from zero gradients."""
        self.lib.check(self.lib.scalar_set_grad_scheme(self.h, int(grad_scheme)))

    # time-step history (field/history.cpp)
    def set_history_size(self, n):
        self.lib.check(self.lib.scalar_set_history_size(self.h, int(n)))

    def update_prev_time_steps(self):
        self.lib.check(self.lib.scalar_update_prev_time_steps(self.h))

    def update(self, values):
        """Scalar::update: history push, new values, face values cleared."""
        v = np.ascontiguousarray(values, dtype=np.float64)
        self.lib.check(self.lib.scalar_update(self.h, _f64p(v)))

    def history(self, index):
        """getHistory(index): values of the time step `index` back (0 = previous), or None."""
        out = np.zeros(self.mesh.n_cells)
        ok = C.c_int32()
        self.lib.check(self.lib.scalar_history(self.h, int(index), _f64p(out), C.byref(ok)))
        return out if ok.value else None

    def to_points(self):
        """cellToPoint of the cell values: one value per mesh vertex."""
        out = np.zeros(self.mesh.n_vertices)
        self.lib.check(self.lib.scalar_to_points(self.h, _f64p(out)))
        return out

    def prev_values(self):
        return self.history(0)

    def prev_prev_values(self):
        return self.history(1)

    def __del__(self):
        if not getattr(self, "_borrowed", True) and getattr(self, "h", None):
            self.lib.scalar_destroy(self.h)
            self.h = None


def _default_bcs(mesh):
    arr = (A.BC * max(1, mesh.info.n_patches))()
    for p in range(mesh.info.n_patches):
        # a field absent from the case has no boundary condition on any patch: asking for a
        # boundary value raises, as BoundaryPatch::getBoundaryCondition does (boundary.cpp:425-444)
        arr[p].kind = A.BC_EMPTY if mesh.case.patch_is_empty[p] else A.BC_UNKNOWN
    return arr


Pressure = Scalar


class Vector:
    """field::Vector / field::Velocity (three component Scalars)."""

    def __init__(self, name, mesh: Mesh, value=(0.0, 0.0, 0.0), grad_scheme=None, bcs=None,
                 _handle=None):
        self.mesh, self.lib, self.name = mesh, mesh.lib, name
        if _handle is None:
            value = np.asarray(value, dtype=np.float64)
            if value.ndim == 1 and value.shape[0] == 3:
                vals = np.repeat(value[:, None], mesh.n_cells, axis=1).reshape(-1).copy()
            else:
                vals = np.ascontiguousarray(value, dtype=np.float64).reshape(-1)
            gs = mesh.case.grad_scheme(name) if grad_scheme is None else grad_scheme
            bcs = mesh.case.bcs(name) if bcs is None else bcs
            self._bcs = bcs
            h = C.c_void_p()
            self.lib.check(self.lib.vector_create(mesh.h, name.encode(), _f64p(vals), gs, bcs,
                                                  C.byref(h)))
            _handle = h
        self.h = _handle

    def _component(self, k):
        # a borrowed handle wrapped on demand; the wrapper keeps this vector alive
        # (no reference cycle, so finalisation order always follows ownership)
        ch = C.c_void_p()
        self.lib.check(self.lib.vector_component(self.h, k, C.byref(ch)))
        return Scalar(self.name + "_" + "xyz"[k], self.mesh, _handle=ch, _owner=self)

    def x(self):
        return self._component(0)

    def y(self):
        return self._component(1)

    def z(self):
        return self._component(2)

    def clone(self):
        h = C.c_void_p()
        self.lib.check(self.lib.vector_clone(self.h, C.byref(h)))
        return Vector(self.name, self.mesh, _handle=h)

    def values(self):
        out = np.zeros(3 * self.mesh.n_cells)
        self.lib.check(self.lib.vector_get_values(self.h, _f64p(out)))
        return out.reshape(3, -1)

    def set_values(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64).reshape(-1)
        self.lib.check(self.lib.vector_set_values(self.h, _f64p(v)))

    def face_flux(self):
        out = np.zeros(self.mesh.n_faces)
        self.lib.check(self.lib.vector_face_flux(self.h, _f64p(out)))
        return out

    def set_face_flux(self, flux):
        """setFaceFluxValues: the n_faces fluxes fluxAtFace returns from now on."""
        f = np.ascontiguousarray(flux, dtype=np.float64)
        if f.size != self.mesh.n_faces:
            raise ValueError("need one flux per face")
        self.lib.check(self.lib.vector_set_face_flux(self.h, _f64p(f)))

    def to_points(self):
        """cellToPoint of the cell values, shape (n_vertices, 3)."""
        out = np.zeros(3 * self.mesh.n_vertices)
        self.lib.check(self.lib.vector_to_points(self.h, _f64p(out)))
        return out.reshape(-1, 3)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.vector_destroy(self.h)
            self.h = None


Velocity = Vector


class Tensor:
    """field::Tensor; values (9, n_cells) SoA or None for the identity."""

    def __init__(self, name, mesh: Mesh, value=None):
        self.mesh, self.lib, self.name = mesh, mesh.lib, name
        vals = None
        if value is not None:
            value = np.asarray(value, dtype=np.float64)
            if value.shape == (3, 3):
                vals = np.repeat(value.reshape(9, 1), mesh.n_cells, axis=1).reshape(-1).copy()
            else:
                vals = np.ascontiguousarray(value, dtype=np.float64).reshape(-1)
        # tensors are immutable through this API: the cell values are kept for export
        self._values = (np.repeat(np.eye(3).reshape(9, 1), mesh.n_cells, axis=1) if vals is None
                        else vals.reshape(9, -1).copy())
        h = C.c_void_p()
        self.lib.check(self.lib.tensor_create(mesh.h, name.encode(), _f64p(vals), C.byref(h)))
        self.h = h

    def values(self):
        """Cell values, shape (9, n_cells); row 3*i+j holds T(i, j)."""
        return self._values.copy()

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.tensor_destroy(self.h)
            self.h = None


# ---- operations and monitors (operations/operations.h, monitor/courant.h) -----
def _adopt_scalar(name, mesh, handle):
    """Wrap a scalar handle created by the library (owned: destroyed with the wrapper)."""
    s = Scalar.__new__(Scalar)
    s.mesh, s.lib, s.name, s._owner, s._borrowed, s.h = mesh, mesh.lib, name, None, False, handle
    return s


class ops:  # noqa: N801  (namespace prism::ops)
    @staticmethod
    def div(U):
        """ops::div (operations.h:84-100): Scalar "div(<name>)" = (sum of signed face
        fluxes) / volume, computed on the device."""
        h = C.c_void_p()
        U.lib.check(U.lib.ops_div(U.h, C.byref(h)))
        return _adopt_scalar(f"div({U.name})", U.mesh, h)

    @staticmethod
    def grad(field, coord=None):
        """ops::grad (operations.h:102-141): of a Scalar, a Vector "grad(<name>)"
        (or, with coord 0/1/2, the Scalar "grad(<name>)_<x|y|z>"); of a Vector, the
        Tensor "grad(<name>)" with column j the gradient of component j."""
        mesh = field.mesh
        if isinstance(field, Scalar):
            g = field.grad()
            if coord is not None:
                name = f"grad({field.name})_{'xyz'[coord]}"
                return Scalar(name, mesh, g[coord], grad_scheme=A.GRAD_LEAST_SQUARES, bcs=_default_bcs(mesh))
            return Vector(f"grad({field.name})", mesh, value=g, grad_scheme=A.GRAD_LEAST_SQUARES,
                          bcs=_default_bcs(mesh))
        if isinstance(field, Vector):
            g = [field._component(k).grad() for k in range(3)]  # g[j][i] = d U_j / d x_i
            t = np.empty((9, mesh.n_cells))
            for i in range(3):
                for j in range(3):
                    t[3 * i + j] = g[j][i]
            return Tensor(f"grad({field.name})", mesh, t)
        raise TypeError("ops.grad needs a Scalar or a Vector")

    @staticmethod
    def rhie_chow(mdot, U, D, p):
        """mdot's face values from U with ops::rhieChowCorrectFace on the interior faces
        (SIMPLE.cpp:136-138, rhie_chow.h:47-63): U.valueAtFace on boundary faces,
        U_f - D_f (grad p_calculated - grad p_averaged) inside; read them back with
        mdot.face_flux()."""
        mdot.lib.check(mdot.lib.rhie_chow(mdot.h, U.h, D.h, p.h))

    @staticmethod
    def symm(a):
        """0.5 (A + A^T) (operations.h:185-187)."""
        a = np.asarray(a, dtype=np.float64)
        return 0.5 * (a + a.T)

    @staticmethod
    def two_symm(a):
        """A + A^T (operations.h:189-191)."""
        a = np.asarray(a, dtype=np.float64)
        return a + a.T

    @staticmethod
    def dev(a):
        """A - tr(A)/3 I (operations.h:193-195)."""
        a = np.asarray(a, dtype=np.float64)
        return a - np.eye(3) * (np.trace(a) / 3.0)

    @staticmethod
    def double_contraction(a, b):
        """sum_ij A_ij B_ij (operations.h:197-199)."""
        return float((np.asarray(a, dtype=np.float64) * np.asarray(b, dtype=np.float64)).sum())


class monitor:  # noqa: N801  (namespace prism::monitor)
    @staticmethod
    def courant_number(mdot, dt):
        """monitor::courantNumber (courant.cpp:7-24): Scalar "Co" = 0.5 dt sum|flux| / V."""
        h = C.c_void_p()
        mdot.lib.check(mdot.lib.courant_number(mdot.h, float(dt), C.byref(h)))
        return _adopt_scalar("Co", mdot.mesh, h)


# ---- schemes (descriptors consumed by Transport) ------------------------------
class _Convection:
    kind = None

    def __init__(self, U, phi):
        self.U, self.phi = U, phi


class convection:  # noqa: N801  (namespace scheme::convection)
    pass


for _name, _code in A.CONV.items():
    setattr(convection, _name, type(_name, (_Convection,), {"code": _code}))
convection.SecondOrderUpwind = convection.LinearUpwind


class diffusion:  # noqa: N801  (namespace scheme::diffusion)
    class NonCorrected:
        corrected = 0

        def __init__(self, kappa, phi, corrector=A.CORR_OVER_RELAXED):
            self.kappa, self.phi, self.corrector = kappa, phi, corrector

    class Corrected(NonCorrected):
        corrected = 1


class temporal:  # noqa: N801  (namespace scheme::temporal)
    class BackwardEuler:
        """scheme::temporal::BackwardEuler(phi, dt) (backward_euler.cpp:62-83)."""
        code = A.TEMPORAL_BACKWARD_EULER

        def __init__(self, phi, dt=1e-5):
            if dt <= 0.0:
                raise ValueError("dt must be positive")
            self.phi, self.dt = phi, float(dt)

    class AdamMoulton(BackwardEuler):
        """scheme::temporal::AdamMoulton(phi, dt) (adam_moulton.cpp:62-107)."""
        code = A.TEMPORAL_ADAM_MOULTON


class source:  # noqa: N801  (namespace scheme::source)
    class ConstantScalar:
        def __init__(self, phi, sign=A.SIGN_POSITIVE):
            self.phi, self.sign = phi, sign

    class Divergence:
        def __init__(self, U, sign=A.SIGN_POSITIVE):
            self.U, self.sign = U, sign

    class Gradient:
        def __init__(self, phi, coord, sign=A.SIGN_POSITIVE):
            self.phi, self.coord, self.sign = phi, coord, sign


class Transport:
    """eqn::Transport(schemes...): the conserved field is the first scheme's field."""

    def __init__(self, *schemes):
        first = schemes[0]
        phi = first.phi
        self.phi, self.lib = phi, phi.lib
        self._keep = list(schemes)
        h = C.c_void_p()
        self.lib.check(self.lib.transport_create(phi.h, C.byref(h)))
        self.h = h
        for s in schemes:
            if isinstance(s, temporal.BackwardEuler):
                self.lib.check(self.lib.transport_add_temporal(self.h, s.code, s.dt))
            elif isinstance(s, _Convection):
                self.lib.check(self.lib.transport_add_convection(self.h, s.code, s.U.h))
            elif isinstance(s, diffusion.NonCorrected):
                ks = s.kappa.h if isinstance(s.kappa, Scalar) else None
                kt = s.kappa.h if isinstance(s.kappa, Tensor) else None
                self.lib.check(self.lib.transport_add_diffusion(self.h, s.corrected, s.corrector,
                                                                ks, kt))
            elif isinstance(s, source.ConstantScalar):
                self.lib.check(self.lib.transport_add_source(self.h, A.SRC_CONSTANT, s.sign,
                                                             s.phi.h, None, 0))
            elif isinstance(s, source.Divergence):
                self.lib.check(self.lib.transport_add_source(self.h, A.SRC_DIVERGENCE, s.sign,
                                                             None, s.U.h, 0))
            elif isinstance(s, source.Gradient):
                self.lib.check(self.lib.transport_add_source(self.h, A.SRC_GRADIENT, s.sign,
                                                             s.phi.h, None, s.coord))
            else:
                raise TypeError(f"unknown scheme {s!r}")

    def field(self):
        return self.phi

    def set_time_step(self, dt):
        """ITemporal::setTimeStep on the equation's temporal scheme."""
        self.lib.check(self.lib.transport_set_time_step(self.h, float(dt)))

    def add_symmetry_handler(self):
        self.lib.check(self.lib.transport_add_symmetry_handler(self.h))

    def set_under_relax_factor(self, f):
        self.lib.check(self.lib.transport_set_urf(self.h, float(f)))

    def update_coeffs(self):
        self.lib.check(self.lib.transport_update_coeffs(self.h))

    def relax(self):
        self.lib.check(self.lib.transport_relax(self.h))

    def zero_out_coeffs(self):
        self.lib.check(self.lib.transport_zero_coeffs(self.h))

    def system(self):
        """(csr values, rhs) of the current A and b."""
        mesh = self.phi.mesh
        vals = np.zeros(max(1, mesh.info.nnz))
        rhs = np.zeros(mesh.n_cells)
        self.lib.check(self.lib.transport_get_system(self.h, _f64p(vals), _f64p(rhs)))
        return vals[: mesh.info.nnz], rhs

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.transport_destroy(self.h)
            self.h = None


Momentum = Transport


# ---- solvers ---------------------------------------------------------------------
@dataclass
class SolverResult:
    iteration: int
    initial_residual: float
    final_residual: float
    converged: bool
    status: int
    krylov_iterations: int
    krylov_rel_residual: float


def _solve_opts(lib, method, precision, n_iter, eps, ref_cell, ref_value, clear, krylov_tol,
                krylov_max_iter, inner_tol, preconditioner=A.PC_AUTO, graph=False):
    o = A.SolveOpts()
    lib.solve_opts_default(C.byref(o))
    o.method, o.precision, o.n_iter, o.eps = method, precision, n_iter, eps
    o.ref_cell = -1 if ref_cell is None else ref_cell
    o.ref_value, o.clear_coeffs = ref_value, 1 if clear else 0
    if krylov_tol:
        o.krylov_tol = krylov_tol
    if krylov_max_iter:
        o.krylov_max_iter = krylov_max_iter
    if inner_tol:
        o.inner_tol = inner_tol
    o.preconditioner = preconditioner
    o.graph = 1 if graph else 0
    return o


class _Solver:
    method = A.SOLVER_BICGSTAB

    def __init__(self, precision=A.PREC_FP64, krylov_tol=0.0, krylov_max_iter=0, inner_tol=0.0,
                 preconditioner="auto", graph=False):
        """graph=True: solves, and the SIMPLE/PRIME/PISO steps driven by this solver, run as one
        CUDA graph launch with device-side solver loops (FP64 BiCGSTAB; the first call on new
        equations runs as usual and builds what the graph uses)."""
        self.graph = graph
        self.precision, self.krylov_tol = precision, krylov_tol
        self.krylov_max_iter, self.inner_tol = krylov_max_iter, inner_tol
        if isinstance(preconditioner, str):
            preconditioner = A.PRECONDITIONERS[preconditioner]
        self.preconditioner = preconditioner

    def opts(self, lib, n_iter=10, eps=1e-7, ref_cell=None, ref_value=0.0, clear_coeffs=True):
        return _solve_opts(lib, self.method, self.precision, n_iter, eps, ref_cell, ref_value,
                           clear_coeffs, self.krylov_tol, self.krylov_max_iter, self.inner_tol,
                           self.preconditioner, self.graph)

    def solve(self, eqn: Transport, n_iter=10, eps=1e-7, ref_cell=None, ref_value=0.0,
              clear_coeffs=True) -> SolverResult:
        """ISolver::solve (numerics/solver.cpp:27-82)."""
        o = self.opts(eqn.lib, n_iter, eps, ref_cell, ref_value, clear_coeffs)
        r = A.SolveResult()
        eqn.lib.check(eqn.lib.solve(eqn.h, C.byref(o), C.byref(r)))
        return SolverResult(r.iterations, r.initial_residual, r.final_residual, bool(r.converged),
                            r.status, r.krylov_iterations, r.krylov_rel_residual)

    def step(self, lib, rowptr, col, values, x, b):
        """ISolver::step on a raw CSR matrix; returns the new x."""
        rowptr = np.ascontiguousarray(rowptr, np.int64)
        col = np.ascontiguousarray(col, np.int64)
        values = np.ascontiguousarray(values, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        x = np.array(x, dtype=np.float64)
        o = self.opts(lib)
        r = A.SolveResult()
        lib.check(lib.solve_csr(len(b), rowptr.ctypes.data_as(A.pi64), col.ctypes.data_as(A.pi64),
                                _f64p(values), _f64p(b), _f64p(x), C.byref(o), C.byref(r)))
        return x


class BiCGSTAB(_Solver):
    method = A.SOLVER_BICGSTAB


class Jacobi(_Solver):
    method = A.SOLVER_JACOBI


class FCG(_Solver):
    """Flexible CG with an FP32 AMG V-cycle (FP64 recurrences), for symmetric positive
    (semi-)definite systems; no counterpart in the reference."""
    method = A.SOLVER_FCG


# ---- pressure-velocity coupling ------------------------------------------------------
@dataclass
class SIMPLEControls:
    momentum_urf: float = 0.7
    momentum_max_iter: int = 3
    momentum_residual: float = 1e-7
    momentum_residual_stop: float = 1e-5
    non_ortho_correctors: int = 2
    pressure_urf: float = 0.3
    pressure_max_iter: int = 5
    pressure_residual: float = 1e-7
    p_ref_cell: Optional[int] = None
    p_ref_value: float = 0.0
    batched_momentum: bool = False  # momentum components solved together in one persistent launch

    def to_c(self):
        c = A.SIMPLEControls()
        for f in dc_fields(self):
            v = getattr(self, f.name)
            setattr(c, f.name, -1 if (f.name == "p_ref_cell" and v is None) else v)
        return c


@dataclass
class PISOControls:
    outer_iterations: int = 1
    momentum_implicit_steps: int = 1
    pressure_correction_steps: int = 2
    momentum_urf: float = 1.0
    momentum_max_iter: int = 3
    momentum_residual: float = 1e-4
    momentum_residual_stop: float = 1e-5
    non_ortho_correctors: int = 2
    pressure_urf: float = 1.0
    pressure_max_iter: int = 5
    pressure_residual: float = 1e-4
    p_ref_cell: Optional[int] = None
    p_ref_value: float = 0.0
    batched_momentum: bool = False

    def to_c(self):
        c = A.PISOControls()
        for f in dc_fields(self):
            v = getattr(self, f.name)
            setattr(c, f.name, -1 if (f.name == "p_ref_cell" and v is None) else v)
        return c


@dataclass
class ReportEntry:
    field_name: str
    n_iterations: int
    initial_residual: float
    final_residual: float
    converged: bool


class _PressureLinked:
    fn = None

    def __init__(self, controls=None, solver: Optional[_Solver] = None):
        self.controls = controls if controls is not None else self.default_controls()
        self.solver = solver if solver is not None else BiCGSTAB()

    def step(self, momentum_predictors, U, mdot, p):
        lib = U.lib
        eqs = (C.c_void_p * len(momentum_predictors))(*[e.h.value for e in momentum_predictors])
        c = self.controls.to_c()
        o = self.solver.opts(lib)
        reps = (A.Report * 64)()
        n = C.c_int32()
        lib.check(getattr(lib, self.fn)(C.byref(c), eqs, len(momentum_predictors), U.h, mdot.h,
                                        p.h, C.byref(o), reps, 64, C.byref(n)))
        return [ReportEntry(r.field_name.decode(), r.n_iterations, r.initial_residual,
                            r.final_residual, bool(r.converged)) for r in reps[: min(n.value, 64)]]


class IncompressibleSIMPLE(_PressureLinked):
    fn = "simple_step"
    default_controls = SIMPLEControls


class PRIME(_PressureLinked):
    fn = "prime_step"
    default_controls = SIMPLEControls


class PISO(_PressureLinked):
    fn = "piso_step"
    default_controls = PISOControls


def needs_pressure_reference(p: Scalar) -> bool:
    out = C.c_int32()
    p.lib.check(p.lib.needs_pressure_reference(p.h, C.byref(out)))
    return bool(out.value)


# ---- steady fixed point and discrete adjoint ------------------------------------------
@dataclass
class FixedPointResult:
    outer_iterations: int
    krylov_iterations: int
    final_change: float
    converged: bool
    status: int


def _fixed_point(r):
    return FixedPointResult(r.outer_iterations, r.krylov_iterations, r.final_change, bool(r.converged), r.status)


def adjoint_forward(eqn: Transport, solver: Optional[_Solver] = None, max_outer=100,
                    outer_tol=1e-13) -> FixedPointResult:
    """Repeat solver.solve(eqn, n_iter=1) until ||phi_k - phi_{k-1}|| <= outer_tol ||phi_k||: the
    steady state R(phi, kappa, v) = 0 whose adjoint adjoint_backward computes."""
    solver = solver or BiCGSTAB()
    o = solver.opts(eqn.lib, n_iter=1, eps=0.0)
    r = A.FixedPointResult()
    eqn.lib.check(eqn.lib.adjoint_forward(eqn.h, C.byref(o), int(max_outer), float(outer_tol), C.byref(r)))
    return _fixed_point(r)


def adjoint_backward(eqn: Transport, dJ_dphi, solver: Optional[_Solver] = None, max_outer=100,
                     outer_tol=1e-13):
    """Discrete adjoint of the steady diffusion eqn at its current field: returns
    (dJ/dkappa per cell, dJ/dv per boundary face, FixedPointResult) for dJ/dphi."""
    solver = solver or BiCGSTAB()
    mesh = eqn.phi.mesh
    dJ = np.ascontiguousarray(dJ_dphi, dtype=np.float64)
    if dJ.shape != (mesh.n_cells,):
        raise ValueError("dJ_dphi must have one value per cell")
    gk = np.zeros(mesh.n_cells)
    gv = np.zeros(max(1, mesh.info.n_boundary_faces))
    o = solver.opts(eqn.lib, n_iter=1, eps=0.0)
    r = A.FixedPointResult()
    eqn.lib.check(eqn.lib.adjoint_backward(eqn.h, _f64p(dJ), _f64p(gk), _f64p(gv), C.byref(o), int(max_outer),
                                           float(outer_tol), C.byref(r)))
    return gk, gv[: mesh.info.n_boundary_faces], _fixed_point(r)


# ---- batched solves ------------------------------------------------------------------
class BatchSolver:
    """Independent equations solved together in one persistent launch
    (prism_batch_solve): solve(eqns) ~ [solver.solve(e, n_iter=1) for e in eqns]."""

    def __init__(self, solver: Optional[_Solver] = None, lib=None):
        self.solver = solver or BiCGSTAB(precision=A.PREC_MIXED)
        self.lib = lib or _default_lib()
        h = C.c_void_p()
        self.lib.check(self.lib.batch_create(C.byref(h)))
        self.h = h

    def solve(self, eqns, eps=1e-7, clear_coeffs=True):
        n = len(eqns)
        arr = (C.c_void_p * n)(*[e.h.value if isinstance(e.h, C.c_void_p) else e.h for e in eqns])
        res = (A.SolveResult * n)()
        o = self.solver.opts(self.lib, n_iter=1, eps=eps, clear_coeffs=clear_coeffs)
        self.lib.check(self.lib.batch_solve(self.h, C.cast(arr, A.PP), n, C.byref(o), res))
        return [SolverResult(r.iterations, r.initial_residual, r.final_residual, bool(r.converged), r.status,
                             r.krylov_iterations, r.krylov_rel_residual) for r in res]

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.batch_destroy(self.h)
            self.h = None
