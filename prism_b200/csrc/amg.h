// amg.h -- aggregation algebraic multigrid preconditioner for BiCGSTAB and flexible CG.
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
    // K-cycle level (Amg::kLevel): second cycle's result, A z1 and the residual r1
    ArenaBuf<double> kz2, kq1, kr1;
    // smoothed restriction of the down-sweep: b_next = Rt b, Rt = P^T (I - omega A D^-1)
    // (the residual of one damped-Jacobi step from zero, restricted), next-level rows x
    // this level's columns: CSR pattern with the sorted A entries each Rt entry sums
    // (rt_seg/rt_src), SELL layout, FP64 / FP32 values
    bool use_rt = false;  // down-sweep by Rt (else pre-smoothing + member-sum restriction)
    int rt_lpr = 1, rt_nslices = 0;
    int64_t rt_nnz = 0;
    ArenaBuf<int> rt_rowptr, rt_erow, rt_col, rt_csr_pos, rt_sl_off, rt_sl_col, rt_seg, rt_src;
    ArenaBuf<int> rt_perm;  // SELL slot row -> row of Rt (rows ordered by length within windows)
    ArenaBuf<double> rt_vals;
    ArenaBuf<float> rt_vals32;
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
    // set by the caller while the matrix values are those of the last setup (the
    // pressure correction's later correctors, the later outer steps of one solve):
    // setup() then keeps the hierarchy's values instead of recomputing the same ones
    bool values_current = false;
    uint64_t generation = 0;  // new process-wide value whenever a buffer of the hierarchy is (re)allocated
    uint64_t reported_generation = 0;  // PRISM_VERBOSE: the generation whose memory was last printed
    int tail = -1;            // first level of the fused coarse tail (-1: every level launches its own kernels)
    // V-cycle smoother weight and coarse-correction factor; the pressure-correction
    // equation of SIMPLE/PRIME/PISO gains from a larger over-correction
    // (forPressure). PRISM_AMG_OMEGA / PRISM_AMG_SCALE override both. flex_scale:
    // the factor of the cycles that precondition flexible CG (the pressure
    // correction: 2.2, measured best of 1.8-3.2 on the 2.1M-cell cavity;
    // PRISM_AMG_FLEX_SCALE overrides it)
    double omega = 0.9, scale = 1.8, flex_scale = 1.8;
    // levels 1..k_levels are K-cycle levels in applyK() (two flexible-CG steps
    // each, instead of one coarse cycle), when they lie above the fused tail and
    // are not the coarsest
    int k_levels = 0;       // the deepest K level (0: none)
    unsigned k_mask = 0;    // bit l: level l is a K level
    ArenaBuf<double> kscal, kpart;  // K-cycle scalars (8 per level), block partials of its reductions
    ArenaBuf<unsigned int> kcount;
    // the pressure-correction equation: over-correction 2.0 in V-cycles and
    // PRISM_AMG_KCYCLE K-cycle levels for the flexible CG solve (default 0: on the
    // 2.1M-cell cavity one or two K levels cut the iterations by 1.7x / 2.5x but the
    // extra coarse-level launches cost more than that saved)
    void forPressure();
    bool kLevel(size_t l) const;

    // Build the hierarchy (first call) or refresh its values (later calls) for
    // the matrix A, whose CSR pattern (device rowptr/col) lists each row's
    // entries in the order of its SELL slots. mixed: also FP32 values.
    void setup(const SellMatrix& A, const int* rowptr, const int* col, bool mixed, cudaStream_t s);
    // FP32 values of the finest level (valid after setup with mixed)
    const float* vals32() const { return levels.empty() ? nullptr : levels[0]->vals32.p; }
    // z = M^-1 r (one V(1,1) cycle); S (optional): skip the work once the solve has stopped
    // sample: time the finest-level kernels when a profiling window is open
    void apply(const double* r, double* z, const KState* S, cudaStream_t s, bool sample = false);
    // flexible: the cycle preconditions flexible CG (flex_scale)
    void apply32(const float* r, float* z, const KState* S, cudaStream_t s, bool flexible = false,
                 bool sample = false);
    // z = B r by one cycle with the K-cycle levels and flex_scale (a variable
    // preconditioner: flexible CG only), FP64
    void applyK(const double* r, double* z, const KState* S, cudaStream_t s, bool sample = false);
};

}  // namespace pb
