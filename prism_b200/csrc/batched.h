// batched.h -- many independent linear solves in one persistent launch.
#pragma once

#include <vector>

#include "common.h"

namespace pb {

// One system of the batch (device pointers, SELL-32 layout of its mesh).
struct BatchSystem {
    int n = 0, nslices = 0;
    int64_t nnz_padded = 0;
    const int* sl_off = nullptr;
    const int* sl_col = nullptr;
    const int* diag_pos = nullptr;
    const double* vals = nullptr;
    const double* b = nullptr;
    double* x = nullptr;
};

struct BatchOut {
    int64_t iterations = 0;  // BiCGSTAB iterations (inner, all passes)
    int32_t passes = 0;      // refinement passes
    double rel_residual = 0; // FP64 ||b - Ax|| / ||b|| at the end
    int32_t status = PRISM_OK;
};

struct BatchTuning {
    int block = 0, lpr = 0;  // 0: not tuned yet
    float ms = 0.f;
};

// Block-diagonal batch of systems with the same patterns across calls: the
// concatenated pattern, the device vectors and the tuned launch shape persist.
struct BatchPlan {
    std::vector<uintptr_t> key;
    int nprob = 0, nslices = 0;
    int64_t nnz = 0;
    std::vector<int64_t> nnz_off;
    std::vector<int> slice0;
    DevBuf<int> slice_prob, prob_slice0, prob_n, sl_off, col, diag;
    DevBuf<double> A64, x64, b64, dinv, cdot;
    DevBuf<float> A32f, r32, r032, p32, v32, s32, t32, d32;
    DevBuf<double> A32d, r64b, r064, p64, v64, s64, t64, d64;  // FP64 inner iterations
    DevBuf<unsigned char> state;  // per-problem solver state
    DevBuf<int> ctl;
    BatchTuning tune[2];  // [0] FP64 inner, [1] FP32 inner
    // per call: the systems' values, right-hand sides and guesses gathered into the
    // concatenated buffers by one kernel (table of source pointers), and the whole
    // call -- gather, set-up, the persistent solve, scatter of the solutions -- kept
    // as one CUDA graph, replayed while the systems' buffers and options are the same
    DevBuf<unsigned char> copy_tab;
    std::vector<uintptr_t> graph_key;
    struct Exec {  // owned executable graph (movable with the plan)
        cudaGraphExec_t g = nullptr;
        Exec() = default;
        Exec(Exec&& o) noexcept : g(o.g) { o.g = nullptr; }
        Exec& operator=(Exec&& o) noexcept {
            if (this != &o) {
                reset();
                g = o.g;
                o.g = nullptr;
            }
            return *this;
        }
        ~Exec() { reset(); }
        void reset() {
            if (g) cudaGraphExecDestroy(g);
            g = nullptr;
        }
    } graph;
};

// Solves every system to ||b - Ax|| <= tol ||b|| (FP64 residual): BiCGSTAB
// inner iterations (FP32 with FP64 dots when mixed, else FP64), Jacobi right
// preconditioning by column scaling, restarted inner solves reducing the
// residual by itol, FP64 iterative refinement between them, all inside one
// cooperative launch. x holds the initial guesses and receives the solutions.
std::vector<BatchOut> solveBatch(const std::vector<BatchSystem>& sys, BatchPlan& plan, bool mixed, double tol,
                                 double itol, int max_inner, int max_pass, long long maxit, cudaStream_t s);

}  // namespace pb
