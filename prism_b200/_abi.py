"""ctypes declarations of the C-ABI in include/prism_b200.h.

The structures and function signatures here mirror the header one to one. They
are generic over the library they are bound to: `bind(lib, prefix)` attaches
argument/return types to every entry point of a loaded shared library whose
symbols carry `prefix` (the sm_100a library exports them as ``prism_*``).
"""
import ctypes as C

# ---- constants (include/prism_b200.h) --------------------------------------
OK, NOT_CONVERGED, BREAKDOWN, NONFINITE, BAD_ARG, CUDA_ERROR = 0, 1, 2, 3, 4, 5
INVALID_MESH, NO_BC_HANDLER, SPIN_TIMEOUT, INTERNAL, OUT_OF_MEMORY = 6, 7, 8, 9, 10

ELEM_LINE, ELEM_TRIANGLE, ELEM_QUAD, ELEM_TETRA, ELEM_WEDGE, ELEM_HEX = 1, 2, 3, 4, 5, 6

BC_EMPTY, BC_FIXED, BC_NOSLIP, BC_SYMMETRY, BC_OUTLET = 0, 1, 2, 3, 4
BC_ZERO_GRADIENT, BC_FIXED_GRADIENT, BC_UNKNOWN = 5, 6, 7
BC_KIND_BY_NAME = {
    "empty": BC_EMPTY, "fixed": BC_FIXED, "no-slip": BC_NOSLIP, "symmetry": BC_SYMMETRY,
    "outlet": BC_OUTLET, "zero-gradient": BC_ZERO_GRADIENT, "fixed-gradient": BC_FIXED_GRADIENT,
}
BCV_NIL, BCV_SCALAR, BCV_VECTOR = 0, 1, 2

GRAD_LEAST_SQUARES, GRAD_GREEN_GAUSS = 0, 1
CONV = {"Upwind": 0, "CentralDifference": 1, "LinearUpwind": 2, "QUICK": 3, "FROMM": 4,
        "MINMOD": 5, "MUSCL": 6, "SMART": 7}
CORR_OVER_RELAXED, CORR_MINIMUM, CORR_ORTHOGONAL = 0, 1, 2
SRC_CONSTANT, SRC_DIVERGENCE, SRC_GRADIENT = 0, 1, 2
SIGN_POSITIVE, SIGN_NEGATIVE = 0, 1
SOLVER_BICGSTAB, SOLVER_JACOBI, SOLVER_FCG = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1
TEMPORAL_BACKWARD_EULER, TEMPORAL_ADAM_MOULTON = 0, 1
PC_AUTO, PC_JACOBI, PC_AMG = 0, 1, 2
PC_AUTO_MIN_ROWS = 32768
PRECONDITIONERS = {"auto": PC_AUTO, "jacobi": PC_JACOBI, "amg": PC_AMG}

STATUS_NAMES = {
    0: "OK", 1: "NOT_CONVERGED", 2: "BREAKDOWN", 3: "NONFINITE", 4: "BAD_ARG", 5: "CUDA_ERROR",
    6: "INVALID_MESH", 7: "NO_BC_HANDLER", 8: "SPIN_TIMEOUT", 9: "INTERNAL", 10: "OUT_OF_MEMORY",
}

P = C.c_void_p
i32, i64, f64 = C.c_int32, C.c_int64, C.c_double
pi32, pi64, pf64 = C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_double)
pchar_p = C.POINTER(C.c_char_p)


class UnvMesh(C.Structure):
    _fields_ = [("n_nodes", i64), ("xyz", pf64), ("n_elements", i64), ("elem_kind", pi32),
                ("elem_offsets", pi64), ("elem_nodes", pi64), ("n_groups", i32),
                ("group_names", pchar_p), ("group_is_vertex", pi32), ("group_offsets", pi64),
                ("group_elements", pi64), ("n_patches", i32), ("patch_names", pchar_p),
                ("patch_is_empty", pi32)]


class MeshInfo(C.Structure):
    _fields_ = [("n_cells", i64), ("n_faces", i64), ("n_boundary_faces", i64),
                ("n_nonempty_boundary_faces", i64), ("nnz", i64), ("n_patches", i32),
                ("n_gs_levels", i32), ("n_vertices", i64), ("n_cell_vertices", i64)]


class MeshExport(C.Structure):
    _fields_ = [("owner", pi64), ("neighbor", pi64), ("face_patch", pi32), ("face_area", pf64),
                ("face_normal", pf64), ("face_center", pf64), ("cell_volume", pf64),
                ("cell_center", pf64), ("cell_face_offsets", pi64), ("cell_faces", pi64),
                ("csr_rowptr", pi64), ("csr_col", pi64), ("patch_face_offsets", pi64),
                ("patch_faces", pi64), ("vertex_coords", pf64), ("cell_vertex_offsets", pi64),
                ("cell_vertices", pi64), ("cell_original", pi64)]


class BC(C.Structure):
    _fields_ = [("kind", i32), ("value_kind", i32), ("value", f64), ("vector", f64 * 3)]


class SolveOpts(C.Structure):
    _fields_ = [("method", i32), ("precision", i32), ("n_iter", i64), ("eps", f64),
                ("ref_cell", i64), ("ref_value", f64), ("clear_coeffs", i32),
                ("krylov_tol", f64), ("krylov_max_iter", i64), ("inner_tol", f64),
                ("preconditioner", i32), ("graph", i32)]


class SolveResult(C.Structure):
    _fields_ = [("iterations", i64), ("initial_residual", f64), ("final_residual", f64),
                ("converged", i32), ("status", i32), ("krylov_iterations", i64),
                ("krylov_rel_residual", f64)]


class SIMPLEControls(C.Structure):
    _fields_ = [("momentum_urf", f64), ("momentum_max_iter", i64), ("momentum_residual", f64),
                ("momentum_residual_stop", f64), ("non_ortho_correctors", i64),
                ("pressure_urf", f64), ("pressure_max_iter", i64), ("pressure_residual", f64),
                ("p_ref_cell", i64), ("p_ref_value", f64), ("batched_momentum", i32)]


class PISOControls(C.Structure):
    _fields_ = [("outer_iterations", i64), ("momentum_implicit_steps", i64),
                ("pressure_correction_steps", i64), ("momentum_urf", f64),
                ("momentum_max_iter", i64), ("momentum_residual", f64),
                ("momentum_residual_stop", f64), ("non_ortho_correctors", i64),
                ("pressure_urf", f64), ("pressure_max_iter", i64), ("pressure_residual", f64),
                ("p_ref_cell", i64), ("p_ref_value", f64), ("batched_momentum", i32)]


class Report(C.Structure):
    _fields_ = [("field_name", C.c_char * 32), ("n_iterations", i64), ("initial_residual", f64),
                ("final_residual", f64), ("converged", i32)]


class FixedPointResult(C.Structure):
    _fields_ = [("outer_iterations", i64), ("krylov_iterations", i64), ("final_change", f64),
                ("converged", i32), ("status", i32)]


class Profile(C.Structure):
    _fields_ = [("fp64_launches", i64), ("fp64_ms", f64), ("fp64_bytes", f64),
                ("fp32_launches", i64), ("fp32_ms", f64), ("fp32_bytes", f64),
                ("kernel_launches", i64),
                ("amg_down_launches", i64), ("amg_down_ms", f64), ("amg_down_bytes", f64),
                ("amg_post_launches", i64), ("amg_post_ms", f64), ("amg_post_bytes", f64),
                ("graph_launches", i64),
                ("amg32_down_launches", i64), ("amg32_down_ms", f64), ("amg32_down_bytes", f64),
                ("amg32_post_launches", i64), ("amg32_post_ms", f64), ("amg32_post_bytes", f64),
                ("fcg_launches", i64), ("fcg_ms", f64), ("fcg_bytes", f64)]


PP = C.POINTER(P)
# name -> (restype, argtypes); every int-returning entry point returns a status.
SIGNATURES = {
    "last_error": (C.c_char_p, []),
    "mesh_from_unv": (C.c_int, [C.POINTER(UnvMesh), PP]),
    "mesh_info": (C.c_int, [P, C.POINTER(MeshInfo)]),
    "mesh_export": (C.c_int, [P, C.POINTER(MeshExport)]),
    "mesh_destroy": (C.c_int, [P]),
    "mesh_reorder": (C.c_int, [P, i32]),
    "scalar_create": (C.c_int, [P, C.c_char_p, pf64, i32, C.POINTER(BC), PP]),
    "scalar_destroy": (C.c_int, [P]),
    "scalar_set_values": (C.c_int, [P, pf64]),
    "scalar_get_values": (C.c_int, [P, pf64]),
    "scalar_set_face_values": (C.c_int, [P, pf64]),
    "scalar_face_values": (C.c_int, [P, pf64]),
    "scalar_grad": (C.c_int, [P, pf64]),
    "scalar_compute_gradients": (C.c_int, [P]),
    "scalar_set_grad_scheme": (C.c_int, [P, i32]),
    "vector_create": (C.c_int, [P, C.c_char_p, pf64, i32, C.POINTER(BC), PP]),
    "vector_clone": (C.c_int, [P, PP]),
    "vector_destroy": (C.c_int, [P]),
    "vector_component": (C.c_int, [P, i32, PP]),
    "vector_set_values": (C.c_int, [P, pf64]),
    "vector_get_values": (C.c_int, [P, pf64]),
    "vector_face_flux": (C.c_int, [P, pf64]),
    "vector_set_face_flux": (C.c_int, [P, pf64]),
    "ops_div": (C.c_int, [P, PP]),
    "courant_number": (C.c_int, [P, f64, PP]),
    "cell_to_point": (C.c_int, [P, pf64, i32, pf64]),
    "scalar_to_points": (C.c_int, [P, pf64]),
    "vector_to_points": (C.c_int, [P, pf64]),
    "tensor_create": (C.c_int, [P, C.c_char_p, pf64, PP]),
    "tensor_destroy": (C.c_int, [P]),
    "rhie_chow": (C.c_int, [P, P, P, P]),
    "transport_create": (C.c_int, [P, PP]),
    "transport_destroy": (C.c_int, [P]),
    "transport_add_convection": (C.c_int, [P, i32, P]),
    "transport_add_diffusion": (C.c_int, [P, i32, i32, P, P]),
    "transport_add_temporal": (C.c_int, [P, i32, f64]),
    "transport_set_time_step": (C.c_int, [P, f64]),
    "scalar_set_history_size": (C.c_int, [P, i32]),
    "scalar_update_prev_time_steps": (C.c_int, [P]),
    "scalar_update": (C.c_int, [P, pf64]),
    "scalar_history": (C.c_int, [P, i32, pf64, pi32]),
    "transport_add_source": (C.c_int, [P, i32, i32, P, P, i32]),
    "transport_add_symmetry_handler": (C.c_int, [P]),
    "transport_set_urf": (C.c_int, [P, f64]),
    "transport_update_coeffs": (C.c_int, [P]),
    "transport_relax": (C.c_int, [P]),
    "transport_zero_coeffs": (C.c_int, [P]),
    "transport_get_system": (C.c_int, [P, pf64, pf64]),
    "solve_opts_default": (None, [C.POINTER(SolveOpts)]),
    "solve": (C.c_int, [P, C.POINTER(SolveOpts), C.POINTER(SolveResult)]),
    "solve_csr": (C.c_int, [i64, pi64, pi64, pf64, pf64, pf64, C.POINTER(SolveOpts),
                            C.POINTER(SolveResult)]),
    "simple_controls_default": (None, [C.POINTER(SIMPLEControls)]),
    "piso_controls_default": (None, [C.POINTER(PISOControls)]),
    "simple_step": (C.c_int, [C.POINTER(SIMPLEControls), PP, i32, P, P, P, C.POINTER(SolveOpts),
                              C.POINTER(Report), i32, pi32]),
    "prime_step": (C.c_int, [C.POINTER(SIMPLEControls), PP, i32, P, P, P, C.POINTER(SolveOpts),
                             C.POINTER(Report), i32, pi32]),
    "piso_step": (C.c_int, [C.POINTER(PISOControls), PP, i32, P, P, P, C.POINTER(SolveOpts),
                            C.POINTER(Report), i32, pi32]),
    "needs_pressure_reference": (C.c_int, [P, pi32]),
    "profile_start": (C.c_int, [i32]),
    "profile_stop": (C.c_int, [C.POINTER(Profile)]),
    "jacobi_step_noalloc": (C.c_int, [i64, P, P, P, P, P, P]),
    "adjoint_forward": (C.c_int, [P, C.POINTER(SolveOpts), i32, f64, C.POINTER(FixedPointResult)]),
    "batch_create": (C.c_int, [C.POINTER(P)]),
    "batch_destroy": (None, [P]),
    "batch_solve": (C.c_int, [P, PP, i32, C.POINTER(SolveOpts), C.POINTER(SolveResult)]),
    "adjoint_backward": (C.c_int, [P, pf64, pf64, pf64, C.POINTER(SolveOpts), i32, f64,
                                   C.POINTER(FixedPointResult)]),
}


class PrismError(RuntimeError):
    """Raised when a C-ABI call returns a non-OK status (the reference raises
    std::runtime_error / error::NonImplementedBoundaryCondition / error::InvalidMesh)."""

    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


GPU_ONLY = {"profile_start", "profile_stop", "jacobi_step_noalloc", "adjoint_forward", "adjoint_backward",
            "batch_create", "batch_destroy", "batch_solve"}


class Bound:
    """Entry points of one loaded library, addressed without their prefix."""

    def __init__(self, lib, prefix, required=None):
        self.lib = lib
        self.prefix = prefix
        names = SIGNATURES if required is None else {k: SIGNATURES[k] for k in required}
        for name, (res, args) in names.items():
            if not hasattr(lib, prefix + name) and name in GPU_ONLY:
                continue
            fn = getattr(lib, prefix + name)
            fn.restype = res
            fn.argtypes = args
            setattr(self, name, fn)

    def check(self, status):
        if status != OK:
            msg = self.last_error()
            raise PrismError(status, msg.decode() if msg else "")
        return status


def bind(lib, prefix):
    return Bound(lib, prefix)


def exported_symbols(prefix):
    """Every symbol the header declares, with the given prefix."""
    extra = ["status_string"]
    return [prefix + n for n in list(SIGNATURES) + extra]
