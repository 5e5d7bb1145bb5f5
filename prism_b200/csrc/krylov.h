// krylov.h -- BiCGSTAB / flexible-CG / Jacobi steps and the scaled residual on a SELL-32 matrix.
#pragma once

#include "common.h"

namespace pb {

// Matrix in SELL-32 layout (see views.h); vals holds the assembled FP64 values.
struct SellMatrix {
    int n = 0, nslices = 0;
    int64_t nnz_padded = 0;
    const int* sl_off = nullptr;
    const int* col = nullptr;
    const int* diag_pos = nullptr;
    const double* vals = nullptr;
    int64_t nnz_csr = 0;  // structural entries (for algorithmic byte counts)
};

// prism_jacobi_step_noalloc: Jacobi sweep on a device CSR matrix using only static scratch
void jacobiStepNoAlloc(int64_t n, const int32_t* rowptr, const int32_t* col, const double* values, const double* b,
                       double* x, cudaStream_t stream);

// Sampled CUDA-event timing of the BiCGSTAB and flexible-CG SpMV launches and
// of the finest-level AMG cycle kernels.
void profileStart(int max_samples);
void profileStop(PrismProfile* out);
enum ProfKind { PROF_SPMV = 0, PROF_AMG_DOWN = 1, PROF_AMG_POST = 2, PROF_FCG_SPMV = 3 };
// Opens a sample (records the start event on s) when a window is open and has
// room: returns its slot, else -1. profEnd(slot) records the end event.
int profBegin(int kind, bool fp32, double bytes, cudaStream_t s);
void profEnd(int slot, cudaStream_t s);

struct Amg;

// Device-resident solver state (one per BiCGSTAB run).
struct KState {
    double rho, alpha, w, beta;
    double rr, bb, tol2, r0sq;
    double ts, tt;
    double rr_update, delta2;  // mixed precision: |r|^2 at the last reliable update, trigger factor^2
    double dq, dr;             // flexible CG: d.(A d) and d.r of the last direction
    long long iter, maxit;
    int done;  // 0 running, 1 converged, 2 max iterations, 3 restart needed, 4 zero rhs, 5 non-finite,
               // 6 reliable update due (mixed precision)
    int reliable;
};

// Workspace owned by a mesh, sized on first use.
struct KrylovWork {
    int n = 0;
    int64_t nnz = 0;
    DevBuf<double> r, r0, p, v, s, t, xs, dinv, tmp;
    DevBuf<double> As;   // column-scaled matrix A D^-1
    DevBuf<float> As32, r32, r032, p32, v32, s32, t32, x32;
    DevBuf<double> r64;  // mixed precision: FP64 true residual at reliable updates
    DevBuf<double> y, z;       // preconditioned directions M^-1 p, M^-1 s (AMG)
    DevBuf<float> y32, z32;
    void ensurePrec(bool mixed);
    DevBuf<double> partials, scal;
    DevBuf<unsigned int> counter;
    DevBuf<KState> state;
    KState* host_state = nullptr;  // pinned
    // one BiCGSTAB iteration captured as a CUDA graph, kept per operand set (key:
    // precision, matrix, vectors, preconditioner), least recently used last out
    struct IterGraph {
        cudaGraphExec_t exec = nullptr;
        std::vector<uintptr_t> key;
        long long kernels = 0;  // kernel nodes per launch
    };
    std::vector<IterGraph> graphs;
    void ensure(int n_pad, int64_t nnz_padded, bool mixed);
    ~KrylovWork();
};

struct KrylovOut {
    long long iterations = 0;
    int status = PRISM_OK;
    double rel_residual = 0.0;
};

// x <- BiCGSTAB solve of A x = b from the guess x, stopping at ||b - A x|| <= tol ||b||.
// precision: PRISM_PREC_FP64 or PRISM_PREC_MIXED. Right preconditioning: Jacobi
// (column scaling) when amg is null, else one V-cycle of amg, whose hierarchy is
// built on first use from the device CSR pattern (rowptr, col) of A and refreshed
// with A's values on every call.
// flexible: FP64 with amg only -- flexible conjugate gradients (Notay 2000, one
// previous direction kept) preconditioned by amg->applyK(), for symmetric
// positive (semi-)definite A (the pressure-correction equation), in place of
// BiCGSTAB; same stopping rule, passes and statuses.
KrylovOut bicgstab(const SellMatrix& A, const double* b, double* x, double tol, long long maxit, int precision,
                   double inner_tol, KrylovWork& w, cudaStream_t s, Amg* amg = nullptr, const int* rowptr = nullptr,
                   const int* col = nullptr, bool flexible = false);
// flexible CG with amg preconditions with an FP32 V-cycle (else with the FP64 cycle)
bool fcgPre32(const Amg* amg);
// x <- x + D^-1 (b - A x)   (numerics/jacobi.cpp:5-9)
void jacobiStep(const SellMatrix& A, const double* b, double* x, KrylovWork& w, cudaStream_t s);
// max|A x - b| / (max|diag(A) x| + eps)   (numerics/solver.cpp:8-24); returns NaN if non-finite values met
double scaledResidual(const SellMatrix& A, const double* b, const double* x, KrylovWork& w, cudaStream_t s);
// max over rows of sum_{j != i} |a_ij| / |a_ii| (inf for a zero diagonal): below 1, Jacobi
// converges at least that fast, whatever the coupling
double offDiagonalRatio(const SellMatrix& A, KrylovWork& w, cudaStream_t s);
// y <- A x (FP64)
void spmv(const SellMatrix& A, const double* x, double* y, cudaStream_t s);
// H-operator of the explicit momentum step: x_new = (b - (A x - diag x)) / diag  (PRIME.cpp:39-56)
void explicitUpdate(const SellMatrix& A, const double* b, const double* x, double* xnew, cudaStream_t s);

// ---- solves inside a CUDA graph ------------------------------------------
// A solve captured into a graph runs its loops on the device: conditional
// WHILE/IF graph nodes repeat the BiCGSTAB iteration, the restarts and the
// accurate-residual passes of bicgstab() and the outer steps of ISolver::solve,
// decided by one-thread controller kernels that read the solver state, so the
// replayed graph needs no host round trip. SolveCtl is the device record of one
// such solve (read back after the graph ran).
struct SolveCtl {
    long long n_iter, outer;       // ISolver::solve: steps allowed / done
    double eps, init_res, cur_res;
    int converged, status;
    long long kmax, maxit_left, krylov_iterations;
    double tol, krylov_rel;
    int phase, pass, restarts, kstatus;
    long long guard;  // controller passes of the current BiCGSTAB solve
};

// Helper streams for the bodies of nested conditional nodes (one per depth).
struct CaptureStreams {
    cudaStream_t s[3] = {nullptr, nullptr, nullptr};
    cudaStream_t at(int depth);
    ~CaptureStreams();
};
// A conditional handle of the graph being captured on s (reset to dflt at every launch).
cudaGraphConditionalHandle createConditional(cudaStream_t s, unsigned dflt);
// Adds a conditional node (cudaGraphCondTypeWhile / If) on handle h after the
// current capture frontier of s and starts capturing its body on body.
void beginConditional(cudaStream_t s, cudaGraphConditionalNodeType type, cudaGraphConditionalHandle h,
                      cudaStream_t body);
void endConditional(cudaStream_t body);
bool capturing(cudaStream_t s);

// Device-controlled pieces of solve(), emitted into the capture on s:
// ctl := ISolver::solve bookkeeping for n_iter steps, eps, kmax, tol
// (and switches on the outer loop's condition)
void emitSolveBegin(SolveCtl* ctl, long long n_iter, double eps, long long kmax, double tol,
                    cudaGraphConditionalHandle outer, cudaStream_t s);
// w.scal := max|A x - b|, max|diag(A) x|, non-finite flag (the scaled residual's parts)
void emitResidual(const SellMatrix& A, const double* b, const double* x, KrylovWork& w, cudaStream_t s);
// ctl->init_res := the scaled residual in w.scal
void emitInitResidual(SolveCtl* ctl, KrylovWork& w, cudaStream_t s);
// one ISolver::solve step's end: ctl->cur_res from w.scal, status, converged,
// outer count; sets the outer loop's condition (continue while not converged
// and outer < n_iter)
void emitOuterStep(SolveCtl* ctl, KrylovWork& w, cudaGraphConditionalHandle outer, cudaStream_t s);
// the FP64 bicgstab() of one step, as device-controlled nodes (streams: helpers for the bodies)
void emitBicgstab(const SellMatrix& A, const double* b, double* x, double tol, long long maxit, KrylovWork& w,
                  cudaStream_t s, Amg* amg, const int* rowptr, const int* col, SolveCtl* ctl, CaptureStreams& cs,
                  int depth, bool flexible = false);

}  // namespace pb
