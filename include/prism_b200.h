/*
 * prism_b200.h -- C-ABI of the B200 (sm_100a) implementation of Prism's
 * finite-volume hot path: mesh flattening, face-loop assembly, gradients,
 * BiCGSTAB/Jacobi and the SIMPLE/PISO/PRIME drivers.
 *
 * Conventions (all entry points):
 *   - every function returns an int status (PRISM_OK == 0) and never throws;
 *     prism_last_error() returns a thread-local message for the last failure;
 *   - handles are opaque and own their device memory; destroy them with the
 *     matching *_destroy function (children before the mesh);
 *   - host buffers passed in are borrowed for the duration of the call only;
 *   - vector fields are exchanged as structure-of-arrays: x[0..n), y[0..n),
 *     z[0..n); tensors as 9 blocks of n values, block (3*i+j) = T(i,j);
 *   - calls on one mesh (and the fields/equations built on it) are not
 *     thread-safe, matching the single-threaded reference; all device work of
 *     one mesh runs on the mesh's CUDA stream.
 *
 * Reference (eigemx/prism) interfaces replaced, by entry point:
 *   prism_mesh_from_unv      mesh/unv.cpp:61-110 UnvToPMeshConverter +
 *                            mesh/pmesh.cpp:10-49 PMesh ctor (face reorder)
 *   prism_scalar_*           field/scalar.h:14-127 field::Scalar
 *   prism_vector_*           field/vector.h:17-101 field::GeneralVector
 *   prism_tensor_*           field/tensor.h:7-38 field::Tensor
 *   prism_scalar_grad        gradient/gradient.h:12-43 IGradient::gradAtCell
 *   prism_transport_*        equation/transport.h:27-97 eqn::Transport
 *   prism_transport_add_*    scheme/convection/convection.h:50-136,
 *                            scheme/diffusion/diffusion.h:42-79,
 *                            scheme/source/{constant_scalar,divergence,gradient}.h,
 *                            equation/symmetry.cpp:54-90
 *   prism_solve              numerics/solver.h:43-49 ISolver::solve
 *                            (BiCGSTAB numerics/bicgstab.cpp:7-9,
 *                             Jacobi numerics/jacobi.cpp:5-9)
 *   prism_solve_csr          numerics/solver.h:49 ISolver::step on a raw matrix
 *   prism_simple_step        algorithm/SIMPLE.cpp:200-216 IncompressibleSIMPLE::step
 *   prism_prime_step         algorithm/PRIME.cpp:11-37 PRIME::step
 *   prism_piso_step          algorithm/PISO.cpp:10-55 PISO::step
 *   prism_needs_pressure_reference  algorithm/SIMPLE.cpp:110-122
 *   prism_mesh_reorder       mesh/reorder.h:9-13 CuthillMckee::reorder
 *   prism_ops_div            operations/operations.h:84-100 ops::div
 *   prism_courant_number     monitor/courant.cpp:7-24 monitor::courantNumber
 *   prism_cell_to_point      export.cpp:73-111 (anonymous) cellToPoint
 */
#ifndef PRISM_B200_H
#define PRISM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define PRISM_OK 0
#define PRISM_NOT_CONVERGED 1 /* Krylov iteration cap reached (reported, not fatal) */
#define PRISM_BREAKDOWN 2     /* BiCGSTAB rho or omega became zero */
#define PRISM_NONFINITE 3     /* NaN/Inf met in the system or the iterate */
#define PRISM_BAD_ARG 4
#define PRISM_CUDA_ERROR 5
#define PRISM_INVALID_MESH 6  /* error::InvalidMesh (exceptions.h:20-27) */
#define PRISM_NO_BC_HANDLER 7 /* error::NonImplementedBoundaryCondition (exceptions.h:9-18) */
#define PRISM_SPIN_TIMEOUT 8  /* a bounded device-side wait expired */
#define PRISM_INTERNAL 9
#define PRISM_OUT_OF_MEMORY 10

/* ---- enumerations ------------------------------------------------------- */
/* element kinds of a UNV element list (unv.cpp:124-160) */
#define PRISM_ELEM_LINE 1
#define PRISM_ELEM_TRIANGLE 2
#define PRISM_ELEM_QUAD 3
#define PRISM_ELEM_TETRA 4
#define PRISM_ELEM_WEDGE 5
#define PRISM_ELEM_HEX 6

/* boundary-condition kinds, i.e. the "type" strings of <field>.json */
#define PRISM_BC_EMPTY 0          /* "empty" */
#define PRISM_BC_FIXED 1          /* "fixed" */
#define PRISM_BC_NOSLIP 2         /* "no-slip" */
#define PRISM_BC_SYMMETRY 3       /* "symmetry" */
#define PRISM_BC_OUTLET 4         /* "outlet" */
#define PRISM_BC_ZERO_GRADIENT 5  /* "zero-gradient" */
#define PRISM_BC_FIXED_GRADIENT 6 /* "fixed-gradient" */
#define PRISM_BC_UNKNOWN 7        /* any other string: no handler registered */

/* value kind of a boundary condition (mesh/boundary.h BoundaryConditionValueKind) */
#define PRISM_BCV_NIL 0
#define PRISM_BCV_SCALAR 1
#define PRISM_BCV_VECTOR 2

#define PRISM_GRAD_LEAST_SQUARES 0 /* gradient/least_squares.cpp */
#define PRISM_GRAD_GREEN_GAUSS 1   /* gradient/green_gauss.cpp */

#define PRISM_CONV_UPWIND 0 /* convection.cpp:89-128 weightsNVF */
#define PRISM_CONV_CENTRAL 1
#define PRISM_CONV_LINEAR_UPWIND 2 /* "SecondOrderUpwind" */
#define PRISM_CONV_QUICK 3
#define PRISM_CONV_FROMM 4
#define PRISM_CONV_MINMOD 5
#define PRISM_CONV_MUSCL 6
#define PRISM_CONV_SMART 7

#define PRISM_CORR_OVER_RELAXED 0 /* nonortho.cpp:7-21 */
#define PRISM_CORR_MINIMUM 1
#define PRISM_CORR_ORTHOGONAL 2

#define PRISM_SRC_CONSTANT 0   /* source::ConstantScalar */
#define PRISM_SRC_DIVERGENCE 1 /* source::Divergence */
#define PRISM_SRC_GRADIENT 2   /* source::Gradient */

#define PRISM_SIGN_POSITIVE 0
#define PRISM_SIGN_NEGATIVE 1

#define PRISM_TEMPORAL_BACKWARD_EULER 0 /* scheme::temporal::BackwardEuler */
#define PRISM_TEMPORAL_ADAM_MOULTON 1   /* scheme::temporal::AdamMoulton */

#define PRISM_SOLVER_BICGSTAB 0
#define PRISM_SOLVER_JACOBI 1
/* flexible conjugate gradients (one previous direction kept) preconditioned by an
 * FP32 AMG V-cycle, FP64 recurrences: for symmetric positive (semi-)definite
 * systems; FP64 precision and the AMG (or automatic) preconditioner only. No
 * counterpart in the reference; SIMPLE/PRIME/PISO use it for the pressure
 * correction on their own. */
#define PRISM_SOLVER_FCG 2

#define PRISM_PREC_FP64 0  /* FP64 Krylov */
#define PRISM_PREC_MIXED 1 /* FP32 BiCGSTAB (FP64 dots) with FP64 reliable updates */

#define PRISM_PC_AUTO 0   /* library choice: AMG from PRISM_PC_AUTO_MIN_ROWS rows, Jacobi below */
#define PRISM_PC_JACOBI 1 /* diagonal (column scaling), the cheapest iteration */
#define PRISM_PC_AMG 2    /* aggregation AMG V-cycle; hierarchy kept per equation, values refreshed per solve */
#define PRISM_PC_AUTO_MIN_ROWS 32768

/* ---- handles ------------------------------------------------------------ */
typedef struct PrismMesh PrismMesh;
typedef struct PrismScalar PrismScalar;
typedef struct PrismVector PrismVector;
typedef struct PrismTensor PrismTensor;
typedef struct PrismTransport PrismTransport;

/* ---- errors --------------------------------------------------------------- */
const char* prism_status_string(int status);
const char* prism_last_error(void);

/* ---- mesh ----------------------------------------------------------------- */
/* A UNV mesh as the converter sees it: nodes, the element list in file order
 * (boundary faces as TRIANGLE/QUAD elements, cells as TETRA/WEDGE/HEX), the
 * element groups (boundary patches) and the patches defined by fields.json in
 * their sorted-name order with their "empty" flag. Node and element indices
 * are 0-based positions in these lists. */
typedef struct {
    int64_t n_nodes;
    const double* xyz; /* 3*n_nodes, interleaved x,y,z */
    int64_t n_elements;
    const int32_t* elem_kind;     /* PRISM_ELEM_* */
    const int64_t* elem_offsets;  /* n_elements+1 */
    const int64_t* elem_nodes;    /* node indices */
    int32_t n_groups;
    const char* const* group_names;
    const int32_t* group_is_vertex; /* 1 for node groups (skipped, unv.cpp:303) */
    const int64_t* group_offsets;   /* n_groups+1 */
    const int64_t* group_elements;  /* element indices */
    int32_t n_patches;
    const char* const* patch_names;
    const int32_t* patch_is_empty;
} PrismUnvMesh;

typedef struct {
    int64_t n_cells;
    int64_t n_faces;
    int64_t n_boundary_faces;
    int64_t n_nonempty_boundary_faces;
    int64_t nnz; /* entries of the CSR pattern (diagonal + face neighbours) */
    int32_t n_patches;
    int32_t n_gs_levels; /* levels of the Green-Gauss in-place sweep schedule */
    int64_t n_vertices;      /* PMesh::vertices(): every UNV node (pmesh.h:40) */
    int64_t n_cell_vertices; /* sum over cells of Cell::verticesIds().size() */
} PrismMeshInfo;

/* Caller-allocated export buffers; any pointer may be NULL. Vectors are SoA. */
typedef struct {
    int64_t* owner;        /* n_faces */
    int64_t* neighbor;     /* n_faces, -1 for boundary faces */
    int32_t* face_patch;   /* n_faces, -1 for interior faces */
    double* face_area;     /* n_faces */
    double* face_normal;   /* 3*n_faces */
    double* face_center;   /* 3*n_faces */
    double* cell_volume;   /* n_cells */
    double* cell_center;   /* 3*n_cells */
    int64_t* cell_face_offsets; /* n_cells+1 */
    int64_t* cell_faces;        /* face ids of each cell, in reference order */
    int64_t* csr_rowptr;        /* n_cells+1 */
    int64_t* csr_col;           /* nnz, column-sorted rows */
    int64_t* patch_face_offsets; /* n_patches+1 */
    int64_t* patch_faces;
    double* vertex_coords;        /* 3*n_vertices */
    int64_t* cell_vertex_offsets; /* n_cells+1 */
    int64_t* cell_vertices;       /* n_cell_vertices: UNV element node order (cell.h:25) */
    int64_t* cell_original;       /* n_cells: each cell's id before prism_mesh_reorder */
} PrismMeshExport;

int prism_mesh_from_unv(const PrismUnvMesh* desc, PrismMesh** out);
int prism_mesh_info(const PrismMesh* mesh, PrismMeshInfo* info);
int prism_mesh_export(const PrismMesh* mesh, PrismMeshExport* out);
int prism_mesh_destroy(PrismMesh* mesh);
/* mesh::CuthillMckee(mesh).reorder(reverse) (mesh/reorder.cpp:8-130): renumbers
 * the cells in (reverse) Cuthill-McKee order -- breadth first from the
 * lowest-degree unvisited cell, neighbours appended by ascending degree, ties
 * as the reference's std::sort leaves them; faces keep their ids and order.
 * Opt-in; call before any field is created on the mesh (PRISM_BAD_ARG after),
 * since field values are indexed by cell id. Volumes follow their cells (the
 * reference's cached volume vector is left in the old order). */
int prism_mesh_reorder(PrismMesh* mesh, int32_t reverse);

/* ---- fields -------------------------------------------------------------- */
/* Boundary condition of one patch for one field (mesh/boundary.h:86-111). */
typedef struct {
    int32_t kind;       /* PRISM_BC_* */
    int32_t value_kind; /* PRISM_BCV_* */
    double value;       /* scalar value */
    double vector[3];   /* vector value */
} PrismBC;

/* values: n_cells (NULL = zeros). bcs: one per patch, in patch order. */
int prism_scalar_create(PrismMesh* mesh, const char* name, const double* values,
                        int32_t grad_scheme, const PrismBC* bcs, PrismScalar** out);
int prism_scalar_destroy(PrismScalar* s);
/* values() = ... (bumps the event number, scalar.cpp:158-162) */
int prism_scalar_set_values(PrismScalar* s, const double* values);
int prism_scalar_get_values(const PrismScalar* s, double* values);
/* setFaceValues (n_faces values) / clearFaceValues when face_values == NULL */
int prism_scalar_set_face_values(PrismScalar* s, const double* face_values);
/* valueAtFace for every face (n_faces); empty-patch faces are written as 0 */
int prism_scalar_face_values(PrismScalar* s, double* out);
/* gradAtCell for every cell (lazy recompute by event number), SoA 3*n_cells */
int prism_scalar_grad(PrismScalar* s, double* grad_out);
/* computeAllCellGradients (forced sweep) */
int prism_scalar_compute_gradients(PrismScalar* s);
/* Scalar::setGradScheme (scalar.cpp:252-258): a new gradient scheme of the given
 * kind (PRISM_GRAD_*) replaces the field's; its gradients start from zero and are
 * recomputed on the next request. A vector's component changes alone (a clone
 * that shared the old scheme keeps it). */
int prism_scalar_set_grad_scheme(PrismScalar* s, int32_t grad_scheme);
/* time-step history (field/history.cpp:1-63): setHistorySize (scalar.cpp:306-308;
 * shrinking drops the oldest steps, 0 clears), updatePrevTimeSteps
 * (scalar.cpp:322-324: the current values become step 0), update (scalar.cpp:
 * 311-320: updatePrevTimeSteps, then values = values, then clearFaceValues) and
 * getHistory (scalar.cpp:336-338: step `index`, 0 = previous time step;
 * *available = 0 and out untouched when there is no such step). */
int prism_scalar_set_history_size(PrismScalar* s, int32_t n_steps);
int prism_scalar_update_prev_time_steps(PrismScalar* s);
int prism_scalar_update(PrismScalar* s, const double* values);
int prism_scalar_history(const PrismScalar* s, int32_t index, double* out, int32_t* available);

/* values: SoA 3*n_cells (NULL = zeros) */
int prism_vector_create(PrismMesh* mesh, const char* name, const double* values,
                        int32_t grad_scheme, const PrismBC* bcs, PrismVector** out);
/* GeneralVector::clone (vector.h:318-336): components share gradient schemes */
int prism_vector_clone(const PrismVector* v, PrismVector** out);
int prism_vector_destroy(PrismVector* v);
/* borrowed component handle (x()/y()/z()) */
int prism_vector_component(PrismVector* v, int32_t coord, PrismScalar** out);
int prism_vector_set_values(PrismVector* v, const double* values);
int prism_vector_get_values(const PrismVector* v, double* values);
/* fluxAtFace for every face (n_faces); empty-patch faces are written as 0 */
int prism_vector_face_flux(PrismVector* v, double* out);
/* GeneralVector::setFaceFluxValues (vector.h:359-377): n_faces fluxes that
 * fluxAtFace returns from now on */
int prism_vector_set_face_flux(PrismVector* v, const double* flux);

/* ---- diagnostics and point data for export ------------------------------ */
/* ops::div (operations/operations.h:84-100,144-169): a new scalar named
 * "div(<name>)" holding, per cell, the signed sum of fluxAtFace over the
 * cell's non-empty faces divided by the cell volume. */
int prism_ops_div(PrismVector* U, PrismScalar** out);
/* monitor::courantNumber (monitor/courant.cpp:7-24): a new scalar named "Co"
 * holding 0.5 * dt * sum(|fluxAtFace|) / volume per cell (empty faces skipped). */
int prism_courant_number(PrismVector* mdot, double dt, PrismScalar** out);
/* output::cellToPoint (export.cpp:73-111): inverse-distance weighted
 * interpolation of cell data to every mesh vertex, weights
 * 1 / max(|x_v - x_c|, DBL_EPSILON) over the cells that use the vertex.
 * cell_data: n_cells*n_components, point_data: n_vertices*n_components, both
 * interleaved per cell / vertex (the VTU layout, not SoA). A vertex that no
 * cell uses fails with PRISM_INVALID_MESH. */
int prism_cell_to_point(PrismMesh* mesh, const double* cell_data, int32_t n_components,
                        double* point_data);
/* cellToPoint of a device-resident field: n_vertices values / 3*n_vertices
 * interleaved x,y,z per vertex (flattenVector order, export.cpp:139-151) */
int prism_scalar_to_points(PrismScalar* s, double* point_data);
int prism_vector_to_points(PrismVector* v, double* point_data);

/* values: 9*n_cells SoA, NULL = identity */
int prism_tensor_create(PrismMesh* mesh, const char* name, const double* values,
                        PrismTensor** out);
int prism_tensor_destroy(PrismTensor* t);

/* ops::rhieChowCorrectFace over a face-value field, as solvePressureEquation
 * applies it (SIMPLE.cpp:136-138, operations/rhie_chow.h:47-63): mdot's face
 * values become U.valueAtFace on every boundary face and the Rhie-Chow corrected
 * U_f - D_f (grad p_f^calculated - grad p_f^averaged) on every interior face, and
 * its face fluxes (read with prism_vector_face_flux) their dot products with the
 * face area vectors. p's gradient is computed first if stale. */
int prism_rhie_chow(PrismVector* mdot, PrismVector* U, PrismTensor* D, PrismScalar* p);

/* ---- equations ------------------------------------------------------------ */
int prism_transport_create(PrismScalar* phi, PrismTransport** out);
int prism_transport_destroy(PrismTransport* eq);
int prism_transport_add_convection(PrismTransport* eq, int32_t scheme, PrismVector* U);
/* exactly one of kappa_scalar / kappa_tensor is non-NULL */
int prism_transport_add_diffusion(PrismTransport* eq, int32_t corrected, int32_t corrector,
                                  PrismScalar* kappa_scalar, PrismTensor* kappa_tensor);
/* CONSTANT: src_scalar; DIVERGENCE: src_vector; GRADIENT: src_scalar + coord */
int prism_transport_add_source(PrismTransport* eq, int32_t kind, int32_t sign,
                               PrismScalar* src_scalar, PrismVector* src_vector, int32_t coord);
/* scheme::temporal::BackwardEuler / AdamMoulton (phi, dt) (backward_euler.cpp:62-86,
 * adam_moulton.cpp:62-107): at most one per equation, in registration order with
 * the other schemes; dt > 0. Assembly needs one history step of the field
 * (two for AdamMoulton's second-order form, one falls back to BackwardEuler). */
int prism_transport_add_temporal(PrismTransport* eq, int32_t kind, double dt);
/* ITemporal::setTimeStep (temporal.cpp:24-31) */
int prism_transport_set_time_step(PrismTransport* eq, double dt);
/* eqn::boundary::Symmetry<Transport> (needs a convection and a diffusion scheme) */
int prism_transport_add_symmetry_handler(PrismTransport* eq);
int prism_transport_set_urf(PrismTransport* eq, double factor);
int prism_transport_update_coeffs(PrismTransport* eq);
int prism_transport_relax(PrismTransport* eq);
int prism_transport_zero_coeffs(PrismTransport* eq);
/* current A (nnz values in the CSR pattern order of prism_mesh_export) and b */
int prism_transport_get_system(const PrismTransport* eq, double* csr_values, double* rhs);

/* ---- solvers ------------------------------------------------------------- */
typedef struct {
    int32_t method;     /* PRISM_SOLVER_* */
    int32_t precision;  /* PRISM_PREC_* (BiCGSTAB only) */
    int64_t n_iter;     /* ISolver::solve n_iter */
    double eps;         /* ISolver::solve eps (scaled residual) */
    int64_t ref_cell;   /* -1: none */
    double ref_value;
    int32_t clear_coeffs;
    double krylov_tol;      /* BiCGSTAB step: stop at ||b-Ax||/||b|| <= krylov_tol (0: default 1e-12) */
    int64_t krylov_max_iter; /* 0: default 2*n_cells */
    double inner_tol;        /* mixed precision: residual reduction between FP64 reliable updates (0: default 0.1) */
    int32_t preconditioner;  /* PRISM_PC_* (BiCGSTAB only) */
    int32_t graph;           /* 1: prism_solve, and the SIMPLE/PRIME/PISO steps given these options, run as
                                one CUDA graph launch whose solver loops (Krylov batches, restarts,
                                accurate-residual passes, outer steps) are device-side conditional
                                nodes, with no host round trip until the end. FP64 BiCGSTAB only; the
                                first call on new equations runs as usual (it builds the AMG
                                hierarchies and work buffers the graph then uses). 0: default. */
} PrismSolveOpts;

typedef struct {
    int64_t iterations; /* outer step() calls, as SolverResult::iteration */
    double initial_residual;
    double final_residual;
    int32_t converged;
    int32_t status;           /* worst Krylov status met (PRISM_OK / NOT_CONVERGED / ...) */
    int64_t krylov_iterations; /* total inner Krylov iterations */
    double krylov_rel_residual; /* ||b-Ax||/||b|| after the last step */
} PrismSolveResult;

void prism_solve_opts_default(PrismSolveOpts* opts);
int prism_solve(PrismTransport* eq, const PrismSolveOpts* opts, PrismSolveResult* result);
/* x <- step(A, x, b) on a raw CSR matrix (host arrays, int64 indices) */
int prism_solve_csr(int64_t n, const int64_t* rowptr, const int64_t* col, const double* values,
                    const double* b, double* x, const PrismSolveOpts* opts,
                    PrismSolveResult* result);

/* ---- pressure-velocity coupling --------------------------------------------- */
typedef struct {
    double momentum_urf;
    int64_t momentum_max_iter;
    double momentum_residual;
    double momentum_residual_stop;
    int64_t non_ortho_correctors;
    double pressure_urf;
    int64_t pressure_max_iter;
    double pressure_residual;
    int64_t p_ref_cell; /* -1: none */
    double p_ref_value;
    int32_t batched_momentum; /* 1: the momentum predictors of a step are solved together in one
                                 persistent launch (prism_batch_*: Jacobi-preconditioned BiCGSTAB
                                 on every component at once) instead of one solve each; not a
                                 reference control, default 0 */
} PrismSIMPLEControls;

typedef struct {
    int64_t outer_iterations;
    int64_t momentum_implicit_steps;
    int64_t pressure_correction_steps;
    double momentum_urf;
    int64_t momentum_max_iter;
    double momentum_residual;
    double momentum_residual_stop;
    int64_t non_ortho_correctors;
    double pressure_urf;
    int64_t pressure_max_iter;
    double pressure_residual;
    int64_t p_ref_cell;
    double p_ref_value;
    int32_t batched_momentum; /* as in PrismSIMPLEControls */
} PrismPISOControls;

typedef struct {
    char field_name[32];
    int64_t n_iterations;
    double initial_residual;
    double final_residual;
    int32_t converged;
} PrismReport;

void prism_simple_controls_default(PrismSIMPLEControls* c);
void prism_piso_controls_default(PrismPISOControls* c);
/* solver_opts may be NULL: FP64 BiCGSTAB with default Krylov settings */
int prism_simple_step(const PrismSIMPLEControls* controls, PrismTransport* const* momentum,
                      int32_t n_momentum, PrismVector* U, PrismVector* mdot, PrismScalar* p,
                      const PrismSolveOpts* solver_opts, PrismReport* reports,
                      int32_t max_reports, int32_t* n_reports);
int prism_prime_step(const PrismSIMPLEControls* controls, PrismTransport* const* momentum,
                     int32_t n_momentum, PrismVector* U, PrismVector* mdot, PrismScalar* p,
                     const PrismSolveOpts* solver_opts, PrismReport* reports,
                     int32_t max_reports, int32_t* n_reports);
int prism_piso_step(const PrismPISOControls* controls, PrismTransport* const* momentum,
                    int32_t n_momentum, PrismVector* U, PrismVector* mdot, PrismScalar* p,
                    const PrismSolveOpts* solver_opts, PrismReport* reports,
                    int32_t max_reports, int32_t* n_reports);
int prism_needs_pressure_reference(PrismScalar* p, int32_t* out);

/* ---- measurement --------------------------------------------------------- */
/* Live timing of the hot solver kernels, sampled with CUDA events on the
 * launching stream while a profiling window is open, with the algorithmic
 * bytes of the sampled launches (nnz: the structural entries of the matrix):
 *   fp64 / fp32: the SpMV inside BiCGSTAB (v = A p), FP64 / FP32 values:
 *       nnz*(value + 4) + 4*(n+1) + 2*n*value (values, columns, row pointers,
 *       x read once, y written once);
 *   fcg: the SpMV of flexible CG (u = A z with the dots z.q, z.u, z.r), FP64
 *       matrix: nnz*12 + 4*(n+1) + (zbytes + 24)*n (z read in the
 *       preconditioner's precision; u written; q, r read);
 *   amg_down / amg_post (FP64 cycle), amg32_down / amg32_post (FP32 cycle):
 *       the AMG cycle's down-sweep and up-sweep kernels on the finest level,
 *       down, by the smoothed restriction Rt = P^T (I - omega A D^-1) (nc rows):
 *             rt_nnz*(value + 4) + 4*(nc+1) + value*(n + nc) (Rt; b read, next
 *             level's b written);
 *       down, by pre-smoothing with the residual (the member sums not sampled):
 *             nnz*(value + 4) + 4*(n+1) + 4*value*n (matrix; b, D^-1 read; x, r
 *             written);
 *       post: nnz*(value + 4) + 4*(n+1) + (3*value + 4)*n + value*nc (matrix;
 *             b, D^-1, aggregate map read, output written; coarse correction
 *             read), one value per row more when x was stored by the down-sweep.
 * Iterations replayed from a CUDA graph are not sampled. No counterpart in the
 * reference. */
typedef struct {
    int64_t fp64_launches;
    double fp64_ms;
    double fp64_bytes;
    int64_t fp32_launches;
    double fp32_ms;
    double fp32_bytes;
    int64_t kernel_launches; /* every kernel this library launched in the window */
    int64_t amg_down_launches;
    double amg_down_ms;
    double amg_down_bytes;
    int64_t amg_post_launches;
    double amg_post_ms;
    double amg_post_bytes;
    int64_t graph_launches; /* solves and steps run as one CUDA graph launch (PrismSolveOpts.graph) */
    int64_t amg32_down_launches;
    double amg32_down_ms;
    double amg32_down_bytes;
    int64_t amg32_post_launches;
    double amg32_post_ms;
    double amg32_post_bytes;
    int64_t fcg_launches;
    double fcg_ms;
    double fcg_bytes;
} PrismProfile;
int prism_profile_start(int32_t max_samples);
int prism_profile_stop(PrismProfile* out);

/* ---- allocation-free Jacobi sweep ------------------------------------------ */
/* For callers that cannot allocate device memory when they need a solver step
 * (host applications that own a fixed device-memory budget and allocate nothing
 * after start-up; time loops that must not synchronize on cudaMalloc/cudaFree).
 * No counterpart in the reference.
 *
 * One Jacobi sweep x <- x + D^-1 (b - A x) on an n x n CSR matrix whose arrays
 * the caller already holds in device memory: rowptr (n+1) and col (nnz) int32,
 * values (nnz), b and x (n) FP64; all are device pointers and x is updated in
 * place. The work is enqueued on `stream` (a cudaStream_t; NULL = the default
 * stream) and the call returns without waiting for it.
 *
 * Nothing is allocated: the out-of-place sweep uses a fixed scratch vector of
 * PRISM_NOALLOC_MAX_ROWS doubles (8 MiB) that every GPU loading the library
 * holds until the process exits; n above that limit is rejected with
 * PRISM_BAD_ARG. The first call on a device, with that device current, looks up
 * the scratch's device address (cudaGetSymbolAddress): make that first call
 * before any stream capture. All calls share the one scratch vector, so calls
 * whose work overlaps on the GPU (different streams, or different host threads)
 * race; serialize them. Every scratch entry a call reads is written earlier in
 * the same call, so nothing has to be cleared between calls. A row without a
 * diagonal entry follows numerics/jacobi.cpp:5-9 (1/0 = inf, so x + inf (b - Ax)
 * there); prism_solve_csr rejects such a matrix with PRISM_BAD_ARG instead. */
#define PRISM_NOALLOC_MAX_ROWS 1048576
int prism_jacobi_step_noalloc(int64_t n, const int32_t* rowptr, const int32_t* col, const double* values,
                              const double* b, double* x, void* stream);

/* ---- batched solves --------------------------------------------------------- */
/* Many independent equations (any meshes on this GPU) solved together: each is
 * assembled and relaxed as in prism_solve, then every system is solved in one
 * persistent launch -- BiCGSTAB with Jacobi preconditioning per system, FP32
 * inner iterations with FP64 dot products (precision PRISM_PREC_MIXED) or FP64
 * ones, each inner solve reducing its residual by inner_tol (default 1e-4 mixed)
 * between FP64 refinement steps, until ||b - Ax|| <= krylov_tol ||b|| (default
 * 1e-12). The launch shape is autotuned on the first call for a set of
 * patterns and kept in the handle with the concatenated pattern, so repeated
 * calls on the same meshes reuse both. results[i] follows prism_solve with
 * n_iter = 1 (iterations = 1, scaled residuals before and after). The method
 * must be PRISM_SOLVER_BICGSTAB and ref_cell -1. No counterpart in the
 * reference. */
typedef struct PrismBatch PrismBatch;
int prism_batch_create(PrismBatch** out);
void prism_batch_destroy(PrismBatch* batch);
int prism_batch_solve(PrismBatch* batch, PrismTransport* const* eqs, int32_t n, const PrismSolveOpts* opts,
                      PrismSolveResult* results);

/* ---- steady fixed point and discrete adjoint ----------------------------- */
/* A forward/backward pair shaped like a torch.autograd.Function for steady
 * diffusion, -div(kappa grad phi) = f with a scalar kappa field, NonCorrected or
 * Corrected diffusion (least-squares gradient), ConstantScalar sources and
 * Fixed / ZeroGradient / FixedGradient / Symmetry / empty patches. No
 * counterpart in the reference, whose users repeat ISolver::solve
 * (numerics/solver.cpp:27-82) until the non-orthogonal correction settles.
 *
 * prism_adjoint_forward repeats prism_solve(eq, opts) -- assembly, relaxation,
 * Krylov solve -- until the relative change ||phi_k - phi_{k-1}|| / ||phi_k||
 * is <= outer_tol (at most max_outer times). At that fixed point
 * R(phi, kappa, v) = A phi - b = 0, v being the Dirichlet face values.
 *
 * prism_adjoint_backward takes dJ/dphi (host, n_cells) for an objective J(phi)
 * and solves the adjoint (dR/dphi)^T lambda = dJ/dphi at the current phi by
 * the transposed deferred correction A^T lambda_{k+1} = dJ/dphi + C^T lambda_k
 * (C: the correction terms' dependence on phi; one transposed BiCGSTAB solve
 * per step, opts select precision-independent FP64 Krylov settings and the
 * preconditioner), stopping like the forward. It writes
 *   dJ_dkappa[c] = dJ/dkappa_c (host, n_cells), and, when dJ_dface != NULL,
 *   dJ_dface[f]  = dJ/dv_f for every boundary face f < n_boundary_faces (the
 *                  value seen by the diffusion Fixed handler and the gradient:
 *                  the face value of prism_scalar_set_face_values, else the
 *                  patch value; 0 on empty patches and faces without a value).
 * The equation's coefficients are cleared on return. PRISM_BAD_ARG for other
 * equations (convection, tensor kappa, Green-Gauss with Corrected, ...). */
typedef struct {
    int64_t outer_iterations;
    int64_t krylov_iterations;
    double final_change;  /* relative change of the last outer step */
    int32_t converged;
    int32_t status;       /* first non-OK Krylov status, else PRISM_OK */
} PrismFixedPointResult;
int prism_adjoint_forward(PrismTransport* eq, const PrismSolveOpts* opts, int32_t max_outer, double outer_tol,
                          PrismFixedPointResult* result);
int prism_adjoint_backward(PrismTransport* eq, const double* dJ_dphi, double* dJ_dkappa, double* dJ_dface,
                           const PrismSolveOpts* opts, int32_t max_outer, double outer_tol,
                           PrismFixedPointResult* result);

#ifdef __cplusplus
}
#endif
#endif /* PRISM_B200_H */
