// runtime.h -- host objects behind the C-ABI handles: the device mesh, fields,
// equations, and the solve / SIMPLE / PRIME / PISO drivers.
#pragma once

#include <limits>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "amg.h"
#include "assemble.h"
#include "batched.h"
#include "common.h"
#include "krylov.h"
#include "mesh_build.h"
#include "pattern.h"
#include "views.h"

namespace pb {

struct Scalar;
struct Tensor;
struct Transport;
struct BatchHandle;

struct Mesh {
    std::unique_ptr<HostMesh> h;
    cudaStream_t stream = nullptr;
    int nc = 0, nf = 0, nb = 0, nne = 0, npatch = 0, n_pad = 0;
    DevBuf<int> owner, nbr, bpatch, ppos, cf_off, cf_face;
    DevBuf<unsigned char> patch_empty;
    DevBuf<double> area, nx, ny, nz, fx, fy, fz, cx, cy, cz, vol, gcw;
    PatternOutput pat;
    // Green-Gauss sweep schedule: cells grouped by dependency level
    DevBuf<int> level_cells;
    std::vector<int> level_off;
    // least-squares operators (built on first use, shared by every field)
    DevBuf<double> ls_pinv, ls_w;
    bool ls_ready = false;
    KrylovWork kw;
    DevBuf<int> cf_twin, tpos;  // adjoint: twin cell-face entries, transpose positions (built on first use)
    DevBuf<double> asm_rec;      // assembly: 4 doubles per cell-face entry (allocated zeroed on first use)
    std::shared_ptr<Amg> p_amg;  // AMG hierarchy of the pressure-correction equation (SIMPLE/PRIME/PISO)
    // pressure-correction objects of SIMPLE/PRIME/PISO, reset on every step instead of
    // re-created (their device buffers stay allocated between steps)
    std::unique_ptr<Scalar> p_corr;
    std::unique_ptr<Tensor> p_D;
    std::unique_ptr<Transport> p_eq;
    DevBuf<double> scratch;  // n_faces doubles for face exports
    // vertex -> cells map and vertex coordinates for point data (built on first use)
    DevBuf<double> vtx;
    DevBuf<int64_t> v2c_off;
    DevBuf<int> v2c_cell;
    bool points_ready = false;
    bool frozen = false;  // fields exist: the cells can no longer be renumbered
    // solves and steps run as one CUDA graph launch (PrismSolveOpts.graph)
    CaptureStreams cs;
    DevBuf<SolveCtl> graph_ctl;
    SolveCtl* graph_host = nullptr;  // pinned copy of graph_ctl
    cudaGraphExec_t graph_exec = nullptr;
    std::unique_ptr<BatchHandle> mom_batch;  // momentum predictors solved together (batched_momentum)

    ~Mesh();
    MeshView view() const;
    SellMatrix matrix(const double* vals) const;
    void ensureLeastSquares();
};

std::unique_ptr<Mesh> createMesh(const PrismUnvMesh* d);
void reorderMesh(Mesh& m, bool reverse);

struct GradState {
    int type = PRISM_GRAD_LEAST_SQUARES;
    DevBuf<double> g;  // 3 * n_pad
    uint64_t computed = std::numeric_limits<uint64_t>::max();
};

struct Scalar {
    Mesh* m = nullptr;
    std::string name;
    int coord = -1;  // component of a vector field
    DevBuf<double> v;
    DevBuf<double> fv;
    bool has_fv = false;
    std::vector<PrismBC> bc;
    DevBuf<int> bc_kind;
    DevBuf<double> bc_val, bc_vec;
    std::shared_ptr<GradState> grad;
    uint64_t event = 0;
    // time-step history (field/history.cpp): hist[0] = previous time step
    size_t hist_max = 0;
    std::vector<DevBuf<double>> hist;
    ScalarView view() const;
};
void setHistorySize(Scalar& s, size_t n);
void updatePrevTimeSteps(Scalar& s);

struct Vector {
    Mesh* m = nullptr;
    std::string name;
    std::shared_ptr<Scalar> c[3];
    DevBuf<double> fd, ff;
    bool has_fd = false, has_ff = false;
    std::vector<PrismBC> bc;
    DevBuf<int> bc_kind;
    DevBuf<double> bc_vec;
    VectorView view() const;
};

struct Tensor {
    Mesh* m = nullptr;
    DevBuf<double> d;
    int diag = 0;
    TensorView view() const { return {d.p, (int64_t)m->n_pad, diag}; }
};

struct Source {
    int kind, sign, coord;
    Scalar* s = nullptr;
    Vector* U = nullptr;
};

struct Transport {
    Scalar* phi = nullptr;
    int has_conv = 0, conv_scheme = 0, has_diff = 0, corrected = 0, corrector = 0, conv_first = 1;
    int has_temporal = 0, temporal_kind = 0;
    double dt = 1e-5;           // ITemporal default (temporal.h:22)
    int nsch = 0, order[3] = {};  // schemes in registration order (SCH_*)
    Vector* U = nullptr;
    Scalar* ks = nullptr;
    Tensor* kt = nullptr;
    std::vector<Source> sources;
    bool symmetry = false;
    double urf = 1.0;
    bool clean = true;
    DevBuf<double> store;  // A, b, bconv and bdiff in one allocation
    DevSlice<double> A, b, bconv, bdiff;
    std::shared_ptr<Amg> amg;  // AMG hierarchy (PRISM_PC_AMG), built on the first solve
    // symmetric positive (semi-)definite matrix (the pressure correction): with AMG,
    // FP64 solves run flexible CG with the K-cycle instead of BiCGSTAB
    bool spd = false;
    // PRISM_PC_AUTO at AMG sizes, decided on the equation's first solve: Jacobi when
    // its matrix is diagonally dominant enough (offDiagonalRatio), else AMG (0: not yet)
    int auto_pc = 0;
    // the next solves assemble the same matrix as the last one (only b changes):
    // its AMG hierarchy keeps its values
    bool matrix_unchanged = false;
    // adjoint: A^T values and the AMG hierarchy of A^T
    DevBuf<double> AT;
    std::shared_ptr<Amg> amg_adj;
    void ensure();
};

// operations (mirroring the reference call structure)
void ensureGradient(Scalar& s);
// mdot's face values: U.valueAtFace on boundary faces, ops::rhieChowCorrectFace on
// interior faces, with the face fluxes
void rhieChowFaces(Vector& mdot, Vector& U, const Tensor& D, Scalar& p);
void computeGradient(Scalar& s);
void updateCoeffs(Transport& eq);
void relax(Transport& eq);
void zeroOutCoeffs(Transport& eq);
PrismSolveResult solve(Transport& eq, const PrismSolveOpts& o);

// diagnostics into device buffers of n_cells values; cellToPoint writes
// n_vertices * ncomp interleaved values, component k of cell c read from
// comp[k][c * stride]
void opsDiv(Vector& U, double* out);
void courantNumber(Vector& mdot, double dt, double* out);
void cellToPoint(Mesh& m, const double* const* comp, int ncomp, int64_t stride, double* out);

struct Report {
    std::string name;
    int64_t n;
    double init, fin;
    bool conv;
};
void simpleStep(const PrismSIMPLEControls& c, std::vector<Transport*>& mom, Vector& U, Vector& mdot, Scalar& p,
                const PrismSolveOpts& so, std::vector<Report>& rep);
void primeStep(const PrismSIMPLEControls& c, std::vector<Transport*>& mom, Vector& U, Vector& mdot, Scalar& p,
               const PrismSolveOpts& so, std::vector<Report>& rep);
void pisoStep(const PrismPISOControls& c, std::vector<Transport*>& mom, Vector& U, Vector& mdot, Scalar& p,
              const PrismSolveOpts& so, std::vector<Report>& rep);
bool needsPressureReference(const Scalar& p);

// PrismSolveOpts.graph: a solve or a SIMPLE/PRIME/PISO step captured into one
// CUDA graph and launched once. Ready when the solver is FP64 BiCGSTAB and the
// equations' coefficient and work buffers, AMG hierarchies and least-squares
// operators exist (built by an earlier ordinary call), since a capture may not
// allocate or wait on the host.
bool graphReady(const Transport& eq, const PrismSolveOpts& o);
// momentum_solved: the step solves the momentum equations (SIMPLE, PISO), not only applies them (PRIME)
bool stepGraphReady(const std::vector<Transport*>& mom, const Vector& U, const Scalar& p, const PrismSolveOpts& so,
                    bool momentum_solved);
PrismSolveResult solveAsGraph(Transport& eq, const PrismSolveOpts& o);
void stepAsGraph(Mesh& m, const std::function<void()>& step, std::vector<Report>& rep);

// Steady fixed point of repeated solve() calls and its discrete adjoint (pure
// diffusion with a scalar kappa). steadySolve repeats solve(eq, o) until the
// relative change of phi is <= outer_tol; adjointBackward solves the transposed
// problem at the current phi for dJ/dphi (host, n cells) and writes dJ/dkappa
// (host, n cells) and dJ/d(boundary face value) (host, n boundary faces, or null).
struct FixedPointOut {
    int64_t outer = 0, krylov = 0;
    double change = 0.0;
    bool converged = false;
    int status = PRISM_OK;
};
FixedPointOut steadySolve(Transport& eq, const PrismSolveOpts& o, int max_outer, double outer_tol);

// Batched ISolver::solve(eq, n_iter = 1): every equation is assembled and
// relaxed on its mesh, then all systems are solved together in one persistent
// launch (batched.h) and each field receives its solution.
struct BatchHandle {
    BatchPlan plan;
    cudaStream_t stream = nullptr;
    ~BatchHandle();
};
std::vector<PrismSolveResult> solveBatch(BatchHandle& h, std::vector<Transport*>& eqs, const PrismSolveOpts& o);
FixedPointOut adjointBackward(Transport& eq, const double* dJ, double* gk, double* gv, const PrismSolveOpts& o,
                              int max_outer, double outer_tol);
void simpleDefaults(PrismSIMPLEControls* c);
void pisoDefaults(PrismPISOControls* c);
void solveDefaults(PrismSolveOpts* o);
// PRISM_PC_AUTO resolved for an n-row system
int choosePreconditioner(int pc, int64_t n);

}  // namespace pb
