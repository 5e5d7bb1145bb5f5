// amg.h -- aggregation algebraic multigrid preconditioner for BiCGSTAB.
#pragma once

#include <memory>
#include <vector>

#include "common.h"
#include "krylov.h"

namespace pb {

// One level of the hierarchy. Level 0 borrows the equation's matrix (pattern of
// the mesh, values of the equation); coarser levels own theirs. Matrices are
// kept both as CSR (setup) and SELL-32 (cycle kernels). Every buffer lives in
// the hierarchy's arena (Amg::arena).
struct AmgLevel {
    int n = 0, nslices = 0;
    int lpr = 1;  // lanes per row of the cycle kernels
    int64_t nnz = 0, sell_nnz = 0;
    // pattern: CSR view and SELL layout; csr_pos[k] = SELL position of CSR entry k
    const int* rowptr = nullptr;
    const int* col = nullptr;
    const int* csr_pos = nullptr;
    const int* sl_off = nullptr;
    const int* sl_col = nullptr;
    const int* diag_pos = nullptr;
    ArenaBuf<int> o_rowptr, o_col, o_csr_pos, o_sl_off, o_sl_col, o_diag_pos;
    // values (SELL layout): level 0 borrows vals64; FP32 copy for mixed precision
    const double* vals = nullptr;
    ArenaBuf<double> o_vals;
    ArenaBuf<float> vals32;
    ArenaBuf<double> dinv;
    ArenaBuf<float> dinv32;
    // restriction to the next level
    ArenaBuf<int> agg;            // fine row -> aggregate
    ArenaBuf<int> m_off, m_idx;   // aggregate -> member rows
    ArenaBuf<int> gal_seg;        // coarse CSR entry m sums sorted fine entries [gal_seg[m], gal_seg[m+1])
    ArenaBuf<int> gal_src;        // SELL position (this level) of each sorted fine entry
    // cycle vectors (FP64 and FP32)
    ArenaBuf<double> b, x, x2, res;
    ArenaBuf<float> b32, x32, x232, res32;
};

struct Amg {
    DevArena arena;  // memory of every level (declared first: released last)
    std::vector<std::unique_ptr<AmgLevel>> levels;
    int coarse_n = 0;
    ArenaBuf<double> coarse_a, coarse_inv;
    ArenaBuf<float> coarse_inv32;
    ArenaBuf<int> coarse_bad;
    bool built = false;
    bool has32 = false;
    uint64_t generation = 0;  // new process-wide value whenever a buffer of the hierarchy is (re)allocated
    int tail = -1;            // first level of the fused coarse tail (-1: every level launches its own kernels)
    // V-cycle smoother weight and coarse-correction factor; the pressure-correction
    // equation of SIMPLE/PRIME/PISO gains from a larger over-correction
    // (forPressure). PRISM_AMG_OMEGA / PRISM_AMG_SCALE override both.
    double omega = 0.9, scale = 1.8;
    void forPressure() { scale = 2.0; }

    // Build the hierarchy (first call) or refresh its values (later calls) for
    // the matrix A, whose CSR pattern (device rowptr/col) lists each row's
    // entries in the order of its SELL slots. mixed: also FP32 values.
    void setup(const SellMatrix& A, const int* rowptr, const int* col, bool mixed, cudaStream_t s);
    // FP32 values of the finest level (valid after setup with mixed)
    const float* vals32() const { return levels.empty() ? nullptr : levels[0]->vals32.p; }
    // z = M^-1 r (one V(1,1) cycle); S (optional): skip the work once the solve has stopped
    // sample: time the finest-level kernels when a profiling window is open
    void apply(const double* r, double* z, const KState* S, cudaStream_t s, bool sample = false);
    void apply32(const float* r, float* z, const KState* S, cudaStream_t s);
};

}  // namespace pb
