// amg.cu -- aggregation algebraic multigrid, used as the BiCGSTAB preconditioner.
//
// The reference preconditions every BiCGSTAB step with Eigen's IncompleteLUT
// (numerics/bicgstab.h:12). A strong preconditioner is what keeps the
// iteration count of the pressure-correction and transport solves small; on a
// GPU the parallel equivalent is algebraic multigrid:
//   * coarsening: double pairwise aggregation (two matching passes per level,
//     ~5x fewer rows per level). Each pass is a handshake matching on the
//     strong edges (w_ij = (|a_ij|+|a_ji|)/sqrt(|a_ii a_jj|) >= 0.5 of the best
//     edge of both rows), taking for every row its strong edge of highest
//     symmetric hash priority; an edge chosen by both ends is matched. After
//     ten rounds an unmatched row joins the aggregate of its strongest matched
//     strong neighbour, or stays single. Deterministic (no atomics, no races).
//   * prolongation: piecewise constant; Galerkin coarse operator A_c = P^T A P
//     built by sorting the fine entries by (aggregate row, aggregate column)
//     once, after which refreshing the values for a new matrix is one
//     segmented sum per coarse entry in a fixed order;
//   * cycle: V(1,1), damped Jacobi (omega = 0.9) smoothing, coarse correction
//     scaled by 1.8, or 2.0 for the pressure correction (unsmoothed aggregation
//     under-corrects; 2.2 when it preconditions flexible CG), dense inverse
//     (single-block Gauss-Jordan with partial pivoting) on the coarsest level.
//     Each level's down-sweep is one SpMV with the smoothed restriction
//     Rt = P^T (I - omega A D^-1): pre-smoothing from zero, residual and
//     restriction at once (Rt has fewer entries than A: an aggregate's rows share
//     columns), and the up-sweep forms the pre-smoothed x = omega D^-1 b where it
//     reads it, so a level costs two launches; Rt's values are refreshed with the
//     Galerkin operators;
//   * K-cycle (applyK, for the flexible-CG solve of the pressure correction):
//     on the levels Amg::kLevel names, the coarse correction is two
//     flexible-CG steps preconditioned by cycles from that level instead of
//     one over-corrected cycle (see k_first_kernel).
// The hierarchy's structure is built once per matrix pattern and reused; every
// solve refreshes the values from the current matrix.
#include <cooperative_groups.h>
#include <cub/cub.cuh>

#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <type_traits>

#include "amg.h"
#include "reduce.cuh"

namespace pb {

namespace {

constexpr int BS = 256;
constexpr int COARSE_MAX = 128;   // stop coarsening at this many rows
constexpr int DENSE_MAX = 160;    // dense inverse of the coarsest level up to this many rows (fits shared memory)
constexpr int MAX_LEVELS = 20;
constexpr int MATCH_ROUNDS = 10;

inline int grid(int64_t n) { return std::max(1, ceil_div(n, BS)); }

__device__ __forceinline__ unsigned long long edgeHash(int i, int j) {
    unsigned long long a = (unsigned long long)min(i, j), b = (unsigned long long)max(i, j);
    unsigned long long h = (a * 0x9E3779B97F4A7C15ull) ^ (b + 0x632BE59BD9B4E019ull);
    h ^= h >> 31;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 29;
    return h;
}

// ---------------------------------------------------------------- setup kernels
__global__ void weights_kernel(int n, const int* rowptr, const int* col, const int* csr_pos, const int* diag_pos,
                               const double* vals, double* w, double* wmax) {
    int i = blockIdx.x * BS + threadIdx.x;
    if (i >= n) return;
    double aii = fabs(vals[diag_pos[i]]);
    double best = 0.0;
    for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
        int j = col[k];
        if (j == i) {
            w[k] = 0.0;
            continue;
        }
        double aij = fabs(vals[csr_pos[k]]), aji = 0.0;
        for (int q = rowptr[j]; q < rowptr[j + 1]; ++q)
            if (col[q] == i) aji = fabs(vals[csr_pos[q]]);
        double ajj = fabs(vals[diag_pos[j]]);
        double d = aii * ajj;
        double wk = d > 0.0 ? (aij + aji) / sqrt(d) : (aij + aji);
        w[k] = wk;
        best = fmax(best, wk);
    }
    wmax[i] = best;
}

__global__ void propose_kernel(int n, const int* rowptr, const int* col, const double* w, const double* wmax,
                               const int* label, int* cand) {
    int i = blockIdx.x * BS + threadIdx.x;
    if (i >= n) return;
    if (label[i] >= 0) {
        cand[i] = -1;
        return;
    }
    int best = -1;
    unsigned long long bp = 0;
    for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
        int j = col[k];
        if (j == i || label[j] >= 0) continue;
        double wk = w[k];
        if (!(wk > 0.0) || wk < 0.5 * wmax[i] || wk < 0.5 * wmax[j]) continue;
        unsigned long long h = edgeHash(i, j);
        if (best < 0 || h > bp || (h == bp && j < best)) {
            best = j;
            bp = h;
        }
    }
    cand[i] = best;
}

__global__ void accept_kernel(int n, const int* cand, int* label) {
    int i = blockIdx.x * BS + threadIdx.x;
    if (i >= n) return;
    int j = cand[i];
    if (j >= 0 && cand[j] == i) label[i] = min(i, j);
}

// After the handshake rounds: an unmatched row joins the aggregate of its
// strongest matched strong neighbour (ties: lower index), else stays single.
// Reads the round labels, writes the final ones (no order dependence).
__global__ void finish_label_kernel(int n, const int* rowptr, const int* col, const double* w, const double* wmax,
                                    const int* label, int* out, int* root) {
    int i = blockIdx.x * BS + threadIdx.x;
    if (i >= n) return;
    int l = label[i];
    if (l < 0) {
        int best = -1;
        double bw = 0.0;
        for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
            int j = col[k];
            if (j == i || label[j] < 0) continue;
            double wk = w[k];
            if (!(wk > 0.0) || wk < 0.5 * wmax[i] || wk < 0.5 * wmax[j]) continue;
            if (best < 0 || wk > bw || (wk == bw && j < best)) {
                best = j;
                bw = wk;
            }
        }
        l = best >= 0 ? label[best] : i;
    }
    out[i] = l;
    root[i] = (l == i) ? 1 : 0;
}

__global__ void agg_kernel(int n, const int* label, const int* rootid, int* agg) {
    int i = blockIdx.x * BS + threadIdx.x;
    if (i < n) agg[i] = rootid[label[i]];
}

__global__ void compose_kernel(int n, const int* agg1, const int* agg2, int* agg) {
    int i = blockIdx.x * BS + threadIdx.x;
    if (i < n) agg[i] = agg2[agg1[i]];
}

__global__ void keys_kernel(int n, const int* rowptr, const int* col, const int* agg, long long nc, long long* keys,
                            int* idx) {
    int i = blockIdx.x * BS + threadIdx.x;
    if (i >= n) return;
    long long ai = agg[i];
    for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
        keys[k] = ai * nc + agg[col[k]];
        idx[k] = k;
    }
}

// smoothed-restriction keys: agg(i) * ncols + j for every entry (i, j)
__global__ void rt_keys_kernel(int n, const int* rowptr, const int* col, const int* agg, long long ncols,
                               long long* keys, int* idx) {
    int i = blockIdx.x * BS + threadIdx.x;
    if (i >= n) return;
    long long ai = agg[i];
    for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
        keys[k] = ai * ncols + col[k];
        idx[k] = k;
    }
}

__global__ void heads_kernel(int64_t m, const long long* keys, int* head) {
    int64_t q = blockIdx.x * (int64_t)BS + threadIdx.x;
    if (q < m) head[q] = (q == 0 || keys[q] != keys[q - 1]) ? 1 : 0;
}

// coarse CSR from sorted keys: seg start, column, row starts; src = fine SELL position
__global__ void coarse_csr_kernel(int64_t m, const long long* keys, const int* head, const int* mid,
                                  const int* idx_sorted, const int* fine_csr_pos, long long nc, int* seg, int* ccol,
                                  int* crowptr, int* src) {
    int64_t q = blockIdx.x * (int64_t)BS + threadIdx.x;
    if (q >= m) return;
    src[q] = fine_csr_pos[idx_sorted[q]];
    if (!head[q]) return;
    int e = mid[q];
    seg[e] = (int)q;
    long long key = keys[q];
    int r = (int)(key / nc);
    ccol[e] = (int)(key % nc);
    if (q == 0 || keys[q - 1] / nc != r) crowptr[r] = e;
}

__global__ void rowlen_slice_kernel(int n, int nslices, const int* rowptr, int* slice_entries) {
    int s = blockIdx.x * BS + threadIdx.x;
    if (s >= nslices) return;
    int w = 0;
    for (int l = 0; l < 32; ++l) {
        int r = s * 32 + l;
        if (r < n) w = max(w, rowptr[r + 1] - rowptr[r]);
    }
    slice_entries[s] = 32 * w;
}

__global__ void sell_fill_kernel(int n, int nslices, const int* rowptr, const int* col, const int* sl_off,
                                 int* sl_col, int* csr_pos, int* diag_pos) {
    int r = blockIdx.x * BS + threadIdx.x;
    if (r >= nslices * 32) return;
    int s = r >> 5, lane = r & 31;
    int base = sl_off[s], width = (sl_off[s + 1] - base) >> 5;
    if (r >= n) {
        for (int j = 0; j < width; ++j) sl_col[base + 32 * j + lane] = 0;
        return;
    }
    int len = rowptr[r + 1] - rowptr[r];
    for (int j = 0; j < width; ++j) {
        int pos = base + 32 * j + lane;
        if (j < len) {
            int c = col[rowptr[r] + j];
            sl_col[pos] = c;
            csr_pos[rowptr[r] + j] = pos;
            if (c == r) diag_pos[r] = pos;
        } else {
            sl_col[pos] = r;
        }
    }
}

__global__ void member_heads_kernel(int n, const int* agg_sorted, int* m_off) {
    int q = blockIdx.x * BS + threadIdx.x;
    if (q >= n) return;
    if (q == 0 || agg_sorted[q] != agg_sorted[q - 1]) m_off[agg_sorted[q]] = q;
}

// SELL position of every CSR entry (entry j of row r sits in slot j of the row)
__global__ void csr_pos_kernel(int n, const int* rowptr, const int* sl_off, int* csr_pos) {
    int r = blockIdx.x * BS + threadIdx.x;
    if (r >= n) return;
    const int base = sl_off[r >> 5] + (r & 31);
    for (int k = rowptr[r]; k < rowptr[r + 1]; ++k) csr_pos[k] = base + 32 * (k - rowptr[r]);
}

__global__ void iota_kernel(int n, int* v) {
    int i = blockIdx.x * BS + threadIdx.x;
    if (i < n) v[i] = i;
}

// coarse values: sum of the sorted fine entries of each coarse entry, in order
__global__ void galerkin_values_kernel(int nnz_c, const int* seg, const int* src, const double* fine_vals,
                                       const int* coarse_csr_pos, double* coarse_vals) {
    int m = blockIdx.x * BS + threadIdx.x;
    if (m >= nnz_c) return;
    double sum = 0.0;
    for (int q = seg[m]; q < seg[m + 1]; ++q) sum += fine_vals[src[q]];
    coarse_vals[coarse_csr_pos[m]] = sum;
}

// smoothed-restriction values, one entry per thread (erow: the entry's row):
// Rt[c, j] = [agg(j) = c] - omega dinv[j] sum_{i in c} a_ij
__global__ void rt_values_kernel(int nnz, const int* __restrict__ erow, const int* __restrict__ col,
                                 const int* __restrict__ seg, const int* __restrict__ src,
                                 const int* __restrict__ csr_pos, const int* __restrict__ agg,
                                 const double* __restrict__ fine_vals, const double* __restrict__ dinv, double omega,
                                 double* __restrict__ out, float* __restrict__ out32) {
    const int e = blockIdx.x * BS + threadIdx.x;
    if (e >= nnz) return;
    double sum = 0.0;
    for (int q = seg[e]; q < seg[e + 1]; ++q) sum += fine_vals[src[q]];
    const int j = col[e];
    const double v = (agg[j] == erow[e] ? 1.0 : 0.0) - omega * dinv[j] * sum;
    out[csr_pos[e]] = v;
    if (out32) out32[csr_pos[e]] = (float)v;
}

// SELL-C-sigma order of the smoothed restriction's rows: within each window of RT_SIGMA
// rows, longest first (a stable sort keeps equal lengths in row order), so that the
// rows sharing a 32-row slice have similar lengths and the slices little padding
constexpr int RT_SIGMA = 256;
__global__ void rt_order_keys_kernel(int n, const int* rowptr, unsigned* keys, int* rows) {
    const int c = blockIdx.x * BS + threadIdx.x;
    if (c >= n) return;
    const int len = min(rowptr[c + 1] - rowptr[c], 255);
    keys[c] = ((unsigned)(c / RT_SIGMA) << 8) | (unsigned)(255 - len);
    rows[c] = c;
}
// slots of each slice in the permuted order: 32 x the longest of its rows
__global__ void rt_slice_len_kernel(int n, int nslices, const int* rowptr, const int* perm, int* slice_entries) {
    const int sl = blockIdx.x * BS + threadIdx.x;
    if (sl >= nslices) return;
    int w = 0;
    for (int l = 0; l < 32; ++l) {
        const int r = sl * 32 + l;
        if (r < n) w = max(w, rowptr[perm[r] + 1] - rowptr[perm[r]]);
    }
    slice_entries[sl] = 32 * w;
}
// slot row r holds row perm[r]; padded slots read column 0 (value 0)
__global__ void rt_fill_kernel(int n, int nslices, const int* rowptr, const int* col, const int* perm,
                               const int* sl_off, int* sl_col, int* csr_pos) {
    const int r = blockIdx.x * BS + threadIdx.x;
    if (r >= nslices * 32) return;
    const int s = r >> 5, lane = r & 31;
    const int base = sl_off[s], width = (sl_off[s + 1] - base) >> 5;
    const int c = r < n ? perm[r] : -1;
    const int len = c >= 0 ? rowptr[c + 1] - rowptr[c] : 0;
    for (int j = 0; j < width; ++j) {
        const int pos = base + 32 * j + lane;
        if (j < len) {
            sl_col[pos] = col[rowptr[c] + j];
            csr_pos[rowptr[c] + j] = pos;
        } else {
            sl_col[pos] = 0;
        }
    }
}

__global__ void entry_rows_kernel(int n, const int* rowptr, int* erow) {
    const int r = blockIdx.x * BS + threadIdx.x;
    if (r >= n) return;
    for (int e = rowptr[r]; e < rowptr[r + 1]; ++e) erow[e] = r;
}

__global__ void dinv_kernel(int n, const int* diag_pos, const double* vals, double* dinv, float* dinv32) {
    int i = blockIdx.x * BS + threadIdx.x;
    if (i >= n) return;
    double d = vals[diag_pos[i]];
    double di = d != 0.0 ? 1.0 / d : 0.0;
    dinv[i] = di;
    if (dinv32) dinv32[i] = (float)di;
}

__global__ void to_float_kernel(int64_t m, const double* a, float* b) {
    for (int64_t k = blockIdx.x * (int64_t)BS + threadIdx.x; k < m; k += (int64_t)gridDim.x * BS) b[k] = (float)a[k];
}

__global__ void dense_fill_kernel(int n, const int* rowptr, const int* col, const int* csr_pos, const double* vals,
                                  double* M) {
    int r = blockIdx.x * BS + threadIdx.x;
    if (r >= n) return;
    for (int j = 0; j < n; ++j) M[(size_t)r * n + j] = 0.0;
    for (int k = rowptr[r]; k < rowptr[r + 1]; ++k) M[(size_t)r * n + col[k]] += vals[csr_pos[k]];
}

// In-place Gauss-Jordan inversion (partial pivoting) of the n x n row-major
// matrix M in shared memory, one block of 32 warps. A pivot below 1e-12 of the
// largest diagonal entry marks a singular direction (e.g. the constant vector
// of an all-Neumann Laplacian): its row and column are zeroed, which yields the
// solution of a consistent system with that unknown set to zero.
__global__ void __launch_bounds__(1024) gauss_jordan_kernel(int n, const double* __restrict__ M,
                                                            double* __restrict__ inv, float* __restrict__ inv32,
                                                            int* __restrict__ nsing) {
    extern __shared__ double a[];
    __shared__ double fac[DENSE_MAX];
    __shared__ int perm[DENSE_MAX];
    __shared__ int red_i[32];
    __shared__ double amax;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (int e = t; e < n * n; e += blockDim.x) a[e] = M[e];
    __syncthreads();
    if (t == 0) {
        double m = 0.0;
        for (int i = 0; i < n; ++i) m = fmax(m, fabs(a[i * n + i]));
        amax = m;
        *nsing = 0;
    }
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        if (warp == 0) {
            double bv = -1.0;
            int bi = k;
            for (int i = k + lane; i < n; i += 32) {
                double v = fabs(a[i * n + k]);
                if (v > bv) {
                    bv = v;
                    bi = i;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                double ov = __shfl_down_sync(0xffffffffu, bv, o);
                int oi = __shfl_down_sync(0xffffffffu, bi, o);
                if (ov > bv || (ov == bv && oi < bi)) {
                    bv = ov;
                    bi = oi;
                }
            }
            if (lane == 0) {
                red_i[0] = bi;
                perm[k] = bi;
            }
        }
        __syncthreads();
        const int p = red_i[0];
        if (p != k)
            for (int j = t; j < n; j += blockDim.x) {
                double x = a[k * n + j];
                a[k * n + j] = a[p * n + j];
                a[p * n + j] = x;
            }
        __syncthreads();
        const double piv = a[k * n + k];
        if (!(fabs(piv) > 1e-12 * amax)) {
            for (int j = t; j < n; j += blockDim.x) {
                a[k * n + j] = 0.0;
                a[j * n + k] = 0.0;
            }
            if (t == 0) *nsing += 1;
            __syncthreads();
            continue;
        }
        for (int i = t; i < n; i += blockDim.x) fac[i] = (i == k) ? 0.0 : a[i * n + k];
        __syncthreads();
        for (int j = t; j < n; j += blockDim.x) a[k * n + j] = (j == k ? 1.0 : a[k * n + j]) / piv;
        __syncthreads();
        for (int i = warp; i < n; i += 32) {
            if (i == k) continue;
            const double f = fac[i];
            for (int j = lane; j < n; j += 32) a[i * n + j] = (j == k ? 0.0 : a[i * n + j]) - f * a[k * n + j];
        }
        __syncthreads();
    }
    for (int k = n - 1; k >= 0; --k) {
        const int p = perm[k];
        if (p != k)
            for (int i = t; i < n; i += blockDim.x) {
                double x = a[i * n + k];
                a[i * n + k] = a[i * n + p];
                a[i * n + p] = x;
            }
        __syncthreads();
    }
    for (int e = t; e < n * n; e += blockDim.x) {
        inv[e] = a[e];
        if (inv32) inv32[e] = (float)a[e];
    }
}

// ---------------------------------------------------------------- cycle kernels
// Row-parallel SELL kernels with LPR lanes per row (LPR divides 32; the lanes
// of a row are adjacent and split its slots round-robin). Coarse levels have
// few, long rows: more lanes per row keep enough loads in flight.

// sum_j A[row, c_j] * xf(c_j); the result is valid in every lane of the row's group
// (a look-ahead of 4 slots per lane measured slower for the post-smoothing kernel).
// CS: the matrix is loaded with the evict-first hint (ld.global.cs), for the finest
// level's restriction Rt, which no other kernel reads: its lines then leave the L2
// first and the vectors stay (level-0 down-sweep of the 2.1M-cell cavity: 28.6 ->
// 23.9 us live). The level-0 A is not hinted: the SpMV that follows the post-smoothing
// shares its column indices, and hinting both kernels made them 1-2% slower.
template <typename T, int LPR, bool CS = false, typename F>
__device__ __forceinline__ T rowSum(const int* __restrict__ sl_off, const int* __restrict__ col,
                                    const T* __restrict__ val, int row, bool valid, int sub, F xf) {
    T sum = 0;
    if (valid) {
        const int s0 = sl_off[row >> 5];
        const int width = (sl_off[(row >> 5) + 1] - s0) >> 5;
        const int bo = s0 + (row & 31);
        for (int j = sub; j < width; j += LPR) {
            const int p = bo + 32 * j;
            if constexpr (CS) sum += __ldcs(val + p) * xf(__ldcs(col + p));
            else sum += val[p] * xf(col[p]);
        }
    }
    if constexpr (LPR > 1) {
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    }
    return sum;
}

// pre-smoothing from zero and residual (the down-sweep of a level without the
// smoothed restriction): x = omega D^-1 b ; res = b - A x, x at the neighbours
// formed on the fly; restrict_kernel then sums the residuals of each aggregate
template <typename T, int LPR>
__global__ void __launch_bounds__(BS) pre_kernel(int n, const int* __restrict__ sl_off, const int* __restrict__ col,
                                                 const T* __restrict__ val, const T* __restrict__ b,
                                                 const T* __restrict__ dinv, T omega, T* __restrict__ x,
                                                 T* __restrict__ res, const KState* S) {
    pdlEnter();
    if (S && S->done) return;
    const int gt = blockIdx.x * BS + threadIdx.x;
    const int row = gt / LPR, sub = gt % LPR;
    const bool valid = row < n;
    const T sum = rowSum<T, LPR>(sl_off, col, val, row, valid, sub, [&](int c) { return omega * dinv[c] * b[c]; });
    if (valid && sub == 0) {
        x[row] = omega * dinv[row] * b[row];
        res[row] = b[row] - sum;
    }
}

template <typename T>
__global__ void restrict_kernel(int nc, const int* m_off, const int* m_idx, const T* res, T* bc, const KState* S) {
    pdlEnter();
    if (S && S->done) return;
    int c = blockIdx.x * BS + threadIdx.x;
    if (c >= nc) return;
    T sum = 0;
    for (int q = m_off[c]; q < m_off[c + 1]; ++q) sum += res[m_idx[q]];
    bc[c] = sum;
}

// down-sweep of a level: the next level's right-hand side bc = Rt b (smoothed
// restriction: pre-smoothing from zero, residual and restriction in one pass); CS on
// the finest level (Rt loaded evict-first, rowSum)
template <typename T, int LPR, bool CS = false>
__global__ void __launch_bounds__(BS) down_kernel(int nc, const int* __restrict__ sl_off, const int* __restrict__ col,
                                                  const T* __restrict__ val, const int* __restrict__ perm,
                                                  const T* __restrict__ b, T* __restrict__ bc, const KState* S) {
    pdlEnter();
    if (S && S->done) return;
    const int gt = blockIdx.x * BS + threadIdx.x;
    const int row = gt / LPR, sub = gt % LPR;  // slot row; it holds row perm[row] of Rt
    const bool valid = row < nc;
    const T sum = rowSum<T, LPR, CS>(sl_off, col, val, row, valid, sub, [&](int j) { return b[j]; });
    if (valid && sub == 0) bc[perm[row]] = sum;
}

// The finer level's xp = x + scale xc[agg] (prolongated correction plus pre-smoothed
// x), written by the coarser level's up-sweep as soon as each coarse value is known:
// xpv[i] = x[i] + scale out[c] for every member i of aggregate c, with x stored by the
// finer level's pre-smoothing or formed as omega D^-1 b. The finer level's up-sweep
// then gathers one vector per slot instead of three.
template <typename T>
struct FineProlong {
    const int* m_off;  // the finer level's aggregates (= this level's rows) -> members
    const int* m_idx;
    const T* x;  // stored pre-smoothed x, or null
    const T* dinv;
    const T* b;
    T omega, scale;
    T* xpv;  // null: nothing to write
};

// prolongation and post-smoothing: out = xp + omega D^-1 (b - A xp), xp = x + scale * xc[agg]
// with x = omega D^-1 b the pre-smoothed solution. XM: 0, x formed where it is read
// (after the smoothed restriction); 1, x stored by pre_kernel; 2, xp precomputed by the
// coarser level (xpv). fp: this level's values prolongated to the finer level (FineProlong).
template <typename T, int LPR, int XM>
__global__ void __launch_bounds__(BS) post_kernel(int n, const int* __restrict__ sl_off, const int* __restrict__ col,
                                                  const T* __restrict__ val, const T* __restrict__ b,
                                                  const T* __restrict__ x, const T* __restrict__ xc,
                                                  const int* __restrict__ agg, T scale, const T* __restrict__ dinv,
                                                  T omega, T* __restrict__ out, const T* __restrict__ xpv,
                                                  const FineProlong<T> fp, const KState* S) {
    pdlEnter();
    if (S && S->done) return;
    const int gt = blockIdx.x * BS + threadIdx.x;
    const int row = gt / LPR, sub = gt % LPR;
    const bool valid = row < n;
    auto xp = [&](int c) {
        if constexpr (XM == 2) return xpv[c];
        else if constexpr (XM == 1) return x[c] + scale * xc[agg[c]];
        else return omega * dinv[c] * b[c] + scale * xc[agg[c]];
    };
    const T sum = rowSum<T, LPR>(sl_off, col, val, row, valid, sub, xp);
    T o = 0;
    if (valid && sub == 0) {
        o = xp(row) + omega * dinv[row] * (b[row] - sum);
        out[row] = o;
    }
    if (fp.xpv) {  // uniform: every lane takes part in the broadcast
        o = __shfl_sync(0xffffffffu, o, (int)(threadIdx.x & 31) & ~(LPR - 1));
        if (valid)
            for (int q = fp.m_off[row] + sub; q < fp.m_off[row + 1]; q += LPR) {
                const int i = fp.m_idx[q];
                const T base = fp.x ? fp.x[i] : fp.omega * fp.dinv[i] * fp.b[i];
                fp.xpv[i] = base + fp.scale * o;
            }
    }
}

// ---- K-cycle (FP64): two flexible-CG steps on a coarse level
// (Notay and Vassilevski 2008, the K-cycle of AGMG). With rc the restricted
// residual and B one cycle from the coarse level:
//   z1 = B rc ; q1 = A z1 ; a1 = (z1.rc)/(z1.q1) ; r1 = rc - a1 q1
//   z2 = B r1 ; gamma = z2.q1 ; beta = z2.(A z2) ; rho2 = z2.r1
//   a2 = rho2 / (beta - gamma^2/(z1.q1)) ; e = (a1 - a2 gamma/(z1.q1)) z1 + a2 z2
// (the second direction is z2 made A-orthogonal to z1); the fine level then
// adds the prolongated e without the V-cycle's over-correction factor. The
// scalars of a level sit in 8 doubles of Amg::kscal.
enum { KS_RHO1 = 0, KS_ALPHA1 = 1, KS_A1 = 2, KS_C1 = 3, KS_C2 = 4, KS_N = 8 };
constexpr int K_MAX_GRID = NUM_SMS * 8;  // reducing K-cycle kernels: grid-stride over at most this many blocks

inline int kGrid(int64_t rows, int lpr) { return std::max(1, std::min<int>(ceil_div(rows * lpr, BS), K_MAX_GRID)); }

// q1 = A z1 ; z1.rc, z1.q1 -> a1
template <int LPR>
__global__ void __launch_bounds__(BS) k_first_kernel(int n, const int* __restrict__ sl_off, const int* __restrict__ col,
                                                     const double* __restrict__ val, const double* __restrict__ z1,
                                                     const double* __restrict__ rc, double* __restrict__ q1,
                                                     double* partials, unsigned int* counter, double* ks,
                                                     const KState* S) {
    pdlEnter();
    if (S && S->done) return;
    const int64_t total = (int64_t)n * LPR;
    double d0 = 0.0, d1 = 0.0;
    for (int64_t base = (int64_t)blockIdx.x * BS; base < total; base += (int64_t)gridDim.x * BS) {
        const int64_t gt = base + threadIdx.x;
        const bool valid = gt < total;
        const int row = (int)(gt / LPR), sub = (int)(gt % LPR);
        const double sum = rowSum<double, LPR>(sl_off, col, val, row, valid, sub, [&](int c) { return z1[c]; });
        if (valid && sub == 0) {
            q1[row] = sum;
            d0 += z1[row] * rc[row];
            d1 += z1[row] * sum;
        }
    }
    double v[2] = {d0, d1}, out[2];
    if (reduceLast<2, false>(v, partials, counter, out) && threadIdx.x == 0) {
        ks[KS_RHO1] = out[0];
        ks[KS_ALPHA1] = out[1];
        ks[KS_A1] = (out[1] > 0.0 && isfinite(out[0])) ? out[0] / out[1] : 0.0;
    }
}

// r1 = rc - a1 q1
__global__ void k_residual_kernel(int n, const double* __restrict__ rc, const double* __restrict__ q1,
                                  const double* __restrict__ ks, double* __restrict__ r1, const KState* S) {
    pdlEnter();
    if (S && S->done) return;
    const double a1 = ks[KS_A1];
    const int i = blockIdx.x * BS + threadIdx.x;
    if (i < n) r1[i] = rc[i] - a1 * q1[i];
}

// z2.q1, z2.(A z2), z2.r1 -> the combination coefficients c1, c2 of z1, z2
// (a non-positive denominator keeps the first step alone: c1 = a1, c2 = 0)
template <int LPR>
__global__ void __launch_bounds__(BS) k_second_kernel(int n, const int* __restrict__ sl_off, const int* __restrict__ col,
                                                      const double* __restrict__ val, const double* __restrict__ z2,
                                                      const double* __restrict__ q1, const double* __restrict__ r1,
                                                      double* partials, unsigned int* counter, double* ks,
                                                      const KState* S) {
    pdlEnter();
    if (S && S->done) return;
    const int64_t total = (int64_t)n * LPR;
    double d0 = 0.0, d1 = 0.0, d2 = 0.0;
    for (int64_t base = (int64_t)blockIdx.x * BS; base < total; base += (int64_t)gridDim.x * BS) {
        const int64_t gt = base + threadIdx.x;
        const bool valid = gt < total;
        const int row = (int)(gt / LPR), sub = (int)(gt % LPR);
        const double sum = rowSum<double, LPR>(sl_off, col, val, row, valid, sub, [&](int c) { return z2[c]; });
        if (valid && sub == 0) {
            const double zi = z2[row];
            d0 += zi * q1[row];
            d1 += zi * sum;
            d2 += zi * r1[row];
        }
    }
    double v[3] = {d0, d1, d2}, out[3];
    if (reduceLast<3, false>(v, partials, counter, out) && threadIdx.x == 0) {
        const double a1 = ks[KS_A1], al1 = ks[KS_ALPHA1];
        double c1 = a1, c2 = 0.0;
        if (al1 > 0.0) {
            const double den = out[1] - out[0] * out[0] / al1;
            const double a2 = out[2] / den;
            if (den > 0.0 && isfinite(a2)) {
                c2 = a2;
                c1 = a1 - a2 * out[0] / al1;
            }
        }
        ks[KS_C1] = c1;
        ks[KS_C2] = c2;
    }
}

// prolongation of a K-cycle correction and post-smoothing:
// out = xp + omega D^-1 (b - A xp), xp = x + (c1 z1 + c2 z2)[agg], x as in post_kernel
template <int LPR, bool SX>
__global__ void __launch_bounds__(BS) post_k_kernel(int n, const int* __restrict__ sl_off, const int* __restrict__ col,
                                                    const double* __restrict__ val, const double* __restrict__ b,
                                                    const double* __restrict__ x, const double* __restrict__ z1,
                                                    const double* __restrict__ z2, const int* __restrict__ agg,
                                                    const double* __restrict__ ks, const double* __restrict__ dinv,
                                                    double omega, double* __restrict__ out, const KState* S) {
    pdlEnter();
    if (S && S->done) return;
    const double c1 = ks[KS_C1], c2 = ks[KS_C2];
    const int gt = blockIdx.x * BS + threadIdx.x;
    const int row = gt / LPR, sub = gt % LPR;
    const bool valid = row < n;
    auto xp = [&](int c) {
        const int a = agg[c];
        if constexpr (SX) return x[c] + (c1 * z1[a] + c2 * z2[a]);
        else return omega * dinv[c] * b[c] + (c1 * z1[a] + c2 * z2[a]);
    };
    const double sum = rowSum<double, LPR>(sl_off, col, val, row, valid, sub, xp);
    if (valid && sub == 0) out[row] = xp(row) + omega * dinv[row] * (b[row] - sum);
}

// damped Jacobi sweep (coarsest level without a dense inverse): out = x + omega D^-1 (b - A x)
template <typename T>
__global__ void smooth0_kernel(int n, T* x, const T* b, const T* dinv, T omega, const KState* S) {
    pdlEnter();
    if (S && S->done) return;
    int i = blockIdx.x * BS + threadIdx.x;
    if (i < n) x[i] = omega * dinv[i] * b[i];
}
template <typename T, int LPR>
__global__ void __launch_bounds__(BS) jacobi_sweep_kernel(int n, const int* __restrict__ sl_off,
                                                          const int* __restrict__ col, const T* __restrict__ val,
                                                          const T* __restrict__ b, const T* __restrict__ x,
                                                          const T* __restrict__ dinv, T omega, T* __restrict__ out,
                                                          const KState* S) {
    pdlEnter();
    if (S && S->done) return;
    const int gt = blockIdx.x * BS + threadIdx.x;
    const int row = gt / LPR, sub = gt % LPR;
    const bool valid = row < n;
    const T sum = rowSum<T, LPR>(sl_off, col, val, row, valid, sub, [&](int c) { return x[c]; });
    if (valid && sub == 0) out[row] = x[row] + omega * dinv[row] * (b[row] - sum);
}

// Calls f(std::integral_constant<int, LPR>) for the level's lanes per row.
template <typename F>
void withLpr(int lpr, F&& f) {
    switch (lpr) {
        case 1: f(std::integral_constant<int, 1>{}); break;
        case 2: f(std::integral_constant<int, 2>{}); break;
        case 4: f(std::integral_constant<int, 4>{}); break;
        case 8: f(std::integral_constant<int, 8>{}); break;
        case 16: f(std::integral_constant<int, 16>{}); break;
        default: f(std::integral_constant<int, 32>{}); break;
    }
}

// Down-sweep of level l (n rows, nnz entries): the smoothed restriction (one launch)
// or pre-smoothing + member-sum restriction (two launches, the smoothed x stored for
// the up-sweep). The coarse levels are latency-bound: one launch fewer wins. On the
// finest level the bytes decide: Rt has about as many entries as A for 3-D stencils
// (C3 128^3: level-0 down 59.6 us against 46.5 + 10 us, and the up-sweep 63 against
// 53.5 us when it forms x itself) and fewer for 2-D ones (the cavity: 23.3 against
// 24.5 + 8 us). PRISM_AMG_RT=0 / 1 forces either on every level.
bool useRestriction(size_t l, int n, int64_t nnz) {
    static const int force = [] {
        const char* e = std::getenv("PRISM_AMG_RT");
        return e && e[0] ? std::atoi(e) : -1;
    }();
    if (force >= 0) return force != 0;
    return l >= 1 || (n > 0 && (double)nnz / n <= 6.0);
}

// lanes per row: enough threads to fill the GPU once, at most the mean row length
// (2, 4 or 8 times as many threads measured slower on the 2.1M-cell cavity)
int lanesPerRow(int n, int64_t nnz) {
    const int64_t target = (int64_t)NUM_SMS * 2048;
    const double mean = n > 0 ? (double)nnz / n : 1.0;
    int l = 1;
    while (l < 32 && (int64_t)n * l * 2 <= target && l < mean) l *= 2;
    return l;
}

// x = Inv b on the coarsest level (one warp per row)
template <typename T>
__global__ void coarse_solve_kernel(int n, const T* __restrict__ inv, const T* __restrict__ b, T* __restrict__ x,
                                    const KState* S) {
    pdlEnter();
    if (S && S->done) return;
    int row = (blockIdx.x * BS + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (row >= n) return;
    T sum = 0;
    for (int c = lane; c < n; c += 32) sum += inv[(size_t)row * n + c] * b[c];
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
    if (lane == 0) x[row] = sum;
}

// coarsest level too large for a dense inverse: a few damped Jacobi sweeps
// ---------------------------------------------------------------- fused coarse tail
// The levels from the first one with at most tailMaxRows() rows down to the
// coarsest run in one launch of a thread-block cluster: the down phases (the
// smoothed restriction, or pre-smoothing with the residual and then the
// restriction), the coarsest solve and the prolongation/post-smoothing phases of
// all those levels are separated by cluster barriers instead of kernel
// boundaries, which on levels this small cost more than the work itself. Rows
// take TAIL_LPR lanes each (slots in order per lane, as in the separate kernels).
// Vectors written inside the launch are read through L2 (ld.global.cg); matrices
// with ordinary loads.
constexpr int TAIL_MAX_LEVELS = 16;
constexpr int TAIL_BS = 1024;

template <typename T>
struct TailLevel {
    int n, nslices;
    const int* sl_off;
    const int* col;
    const T* val;
    const T* dinv;
    const int* agg;    // row -> aggregate of the next level
    const int* m_off;  // aggregate -> member rows (restriction to the next level)
    const int* m_idx;
    const int* rt_sl_off;  // smoothed restriction to the next level (TailParams::rt), slot rows
    const int* rt_col;     // in the order rt_perm gives
    const T* rt_val;
    const int* rt_perm;
    T *b, *x, *x2, *res;
};
template <typename T>
struct TailParams {
    int nlev;      // levels in the tail, the last being the coarsest
    const T* b0;   // right-hand side of the first tail level (its result goes to L[0].x2)
    const T* inv;  // dense inverse of the coarsest level, or null for Jacobi sweeps
    T omega, scale;
    const KState* S;
    int rt;  // every level but the coarsest has its smoothed restriction: one down phase per level
    TailLevel<T> L[TAIL_MAX_LEVELS];
};

// Rows of a tail level, TAIL_LPR lanes per row (the lanes-per-row split of the
// separate kernels on such levels): f(row, valid, sub) for every row, with a
// loop bound uniform across each warp so that the row sums can shuffle.
constexpr int TAIL_LPR = 8;
template <typename F>
__device__ __forceinline__ void tailRows(int n, int g, int nthreads, F f) {
    constexpr int RPW = 32 / TAIL_LPR;  // rows per warp
    const int lane = g & 31;
    for (int rb = (g >> 5) * RPW; rb < n; rb += (nthreads >> 5) * RPW) {
        const int row = rb + lane / TAIL_LPR;
        f(row, row < n, lane % TAIL_LPR);
    }
}

template <typename T>
__global__ void __launch_bounds__(TAIL_BS) tail_kernel(const __grid_constant__ TailParams<T> P) {
    pdlEnter();
    if (P.S && P.S->done) return;  // uniform: the state does not change during this launch
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const int nthreads = (int)cl.num_blocks() * TAIL_BS;
    const int g = (int)cl.block_rank() * TAIL_BS + threadIdx.x;
    const int lane = threadIdx.x & 31, gw = g >> 5, nw = nthreads >> 5;
    const T omega = P.omega, scale = P.scale;
    // down: the next level's right-hand side by the smoothed restriction (one phase), or
    // pre-smoothing from zero with the residual, then restriction (two phases)
    for (int l = 0; l + 1 < P.nlev; ++l) {
        const TailLevel<T>& L = P.L[l];
        const T* b = l == 0 ? P.b0 : L.b;
        const TailLevel<T>& N = P.L[l + 1];
        if (P.rt) {
            tailRows(N.n, g, nthreads, [&](int c, bool valid, int sub) {
                const T sum = rowSum<T, TAIL_LPR>(L.rt_sl_off, L.rt_col, L.rt_val, c, valid, sub,
                                                  [&](int j) { return __ldcg(b + j); });
                if (valid && sub == 0) N.b[L.rt_perm[c]] = sum;
            });
            cl.sync();
            continue;
        }
        tailRows(L.n, g, nthreads, [&](int row, bool valid, int sub) {
            const T sum = rowSum<T, TAIL_LPR>(L.sl_off, L.col, L.val, row, valid, sub,
                                              [&](int c) { return omega * L.dinv[c] * __ldcg(b + c); });
            if (valid && sub == 0) {
                const T br = __ldcg(b + row);
                L.x[row] = omega * L.dinv[row] * br;
                L.res[row] = br - sum;
            }
        });
        cl.sync();
        tailRows(N.n, g, nthreads, [&](int c, bool valid, int sub) {
            T sum = 0;
            if (valid)
                for (int q = L.m_off[c] + sub; q < L.m_off[c + 1]; q += TAIL_LPR) sum += __ldcg(L.res + L.m_idx[q]);
#pragma unroll
            for (int o = TAIL_LPR / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
            if (valid && sub == 0) N.b[c] = sum;
        });
        cl.sync();
    }
    // coarsest level
    {
        const TailLevel<T>& C = P.L[P.nlev - 1];
        const T* b = P.nlev == 1 ? P.b0 : C.b;
        if (P.inv) {
            for (int row = gw; row < C.n; row += nw) {
                T sum = 0;
                for (int c = lane; c < C.n; c += 32) sum += P.inv[(size_t)row * C.n + c] * __ldcg(b + c);
                for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
                if (lane == 0) C.x2[row] = sum;
            }
        } else {
            for (int r = g; r < C.n; r += nthreads) C.x[r] = omega * C.dinv[r] * __ldcg(b + r);
            T* cur = C.x;
            T* nxt = C.res;
            for (int k = 0; k < 8; ++k) {
                cl.sync();
                T* dst = k == 7 ? C.x2 : nxt;
                tailRows(C.n, g, nthreads, [&](int row, bool valid, int sub) {
                    const T sum = rowSum<T, TAIL_LPR>(C.sl_off, C.col, C.val, row, valid, sub,
                                                      [&](int c) { return __ldcg(cur + c); });
                    if (valid && sub == 0) dst[row] = __ldcg(cur + row) + omega * C.dinv[row] * (__ldcg(b + row) - sum);
                });
                nxt = cur;
                cur = dst;
            }
        }
        cl.sync();
    }
    // up: prolongation and post-smoothing
    for (int l = P.nlev - 2; l >= 0; --l) {
        const TailLevel<T>& L = P.L[l];
        const T* xc = P.L[l + 1].x2;
        const T* b = l == 0 ? P.b0 : L.b;
        // the pre-smoothed x = omega D^-1 b: stored by the pre-smoothing phase, or formed here
        auto xp = [&](int c) {
            const T xs = P.rt ? omega * L.dinv[c] * __ldcg(b + c) : __ldcg(L.x + c);
            return xs + scale * __ldcg(xc + L.agg[c]);
        };
        tailRows(L.n, g, nthreads, [&](int row, bool valid, int sub) {
            const T sum = rowSum<T, TAIL_LPR>(L.sl_off, L.col, L.val, row, valid, sub, xp);
            if (valid && sub == 0) L.x2[row] = xp(row) + omega * L.dinv[row] * (__ldcg(b + row) - sum);
        });
        if (l > 0) cl.sync();
    }
}

// rows of the largest level run in the fused tail (PRISM_AMG_TAIL_ROWS; 0 disables it)
int tailMaxRows() {
    static const int v = [] {
        const char* e = std::getenv("PRISM_AMG_TAIL_ROWS");
        return e && e[0] ? std::max(0, std::atoi(e)) : 4096;
    }();
    return v;
}

// CTAs per tail cluster: 16 (a non-portable size) where the device can place
// such a cluster, else the portable 8
template <typename T>
int tailCluster() {
    static const int c = [] {
        int cl = 8;
        if (cudaFuncSetAttribute(tail_kernel<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
            cudaLaunchConfig_t cfg{};
            cfg.gridDim = dim3(16);
            cfg.blockDim = dim3(TAIL_BS);
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = 16;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            int n = 0;
            if (cudaOccupancyMaxActiveClusters(&n, tail_kernel<T>, &cfg) == cudaSuccess && n >= 1) cl = 16;
        }
        cudaGetLastError();  // a refused query leaves no sticky error
        return cl;
    }();
    return c;
}

template <typename T>
void launchTail(const TailParams<T>& P, cudaStream_t s) {
    const int cl = tailCluster<T>();
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)cl);
    cfg.blockDim = dim3(TAIL_BS);
    cfg.stream = s;
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[1].val.programmaticStreamSerializationAllowed = pdlEnabled() ? 1 : 0;
    cfg.attrs = at;
    cfg.numAttrs = 2;
    PB_CUDA(cudaLaunchKernelEx(&cfg, tail_kernel<T>, P));
    countLaunch();
}

// ---------------------------------------------------------------- structure builders
// Handshake pairwise matching on level L: writes the aggregate of every row
// into agg (n entries) and returns the number of aggregates.
int matchPairs(const AmgLevel& L, int* agg, cudaStream_t s) {
    const int n = L.n;
    TmpBuf<double> w(std::max<int64_t>(L.nnz, 1), s), wmax(n, s);
    TmpBuf<int> label(n, s), cand(n, s), root(n + 1, s), rootid(n + 1, s);
    weights_kernel<<<grid(n), BS, 0, s>>>(n, L.rowptr, L.col, L.csr_pos, L.diag_pos, L.vals, w.p, wmax.p); countLaunch();
    PB_CUDA(cudaMemsetAsync(label.p, 0xff, n * sizeof(int), s));
    for (int round = 0; round < MATCH_ROUNDS; ++round) {
        propose_kernel<<<grid(n), BS, 0, s>>>(n, L.rowptr, L.col, w.p, wmax.p, label.p, cand.p); countLaunch();
        accept_kernel<<<grid(n), BS, 0, s>>>(n, cand.p, label.p); countLaunch();
    }
    finish_label_kernel<<<grid(n), BS, 0, s>>>(n, L.rowptr, L.col, w.p, wmax.p, label.p, cand.p, root.p); countLaunch();
    PB_CUDA(cudaMemsetAsync(root.p + n, 0, sizeof(int), s));
    size_t tb = 0;
    PB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, root.p, rootid.p, n + 1, s));
    TmpBuf<unsigned char> tmp(std::max<size_t>(tb, 1), s);
    PB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb, root.p, rootid.p, n + 1, s));
    agg_kernel<<<grid(n), BS, 0, s>>>(n, cand.p, rootid.p, agg); countLaunch();
    int nc = 0;
    PB_CUDA(cudaMemcpyAsync(&nc, rootid.p + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
    PB_LAUNCH("amg matching");
    return nc;
}

// Galerkin structure of P^T A P for the aggregate map `agg` (nc aggregates):
// fills the restriction data of L and creates the coarse level C (pattern + SELL).
void galerkinStructure(DevArena& ar, AmgLevel& L, const int* agg, int nc, AmgLevel& C, cudaStream_t s) {
    const int n = L.n;
    const int64_t m = L.nnz;
    TmpBuf<long long> keys(m, s), keys_s(m, s);
    TmpBuf<int> idx(m, s), idx_s(m, s), head(m + 1, s), mid(m + 1, s);
    keys_kernel<<<grid(n), BS, 0, s>>>(n, L.rowptr, L.col, agg, nc, keys.p, idx.p); countLaunch();
    int end_bit = 1;
    while (end_bit < 63 && ((long long)1 << end_bit) < (long long)nc * nc) ++end_bit;
    size_t tb = 0;
    PB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.p, keys_s.p, idx.p, idx_s.p, m, 0, end_bit, s));
    TmpBuf<unsigned char> tmp(std::max<size_t>(tb, 1), s);
    PB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, keys.p, keys_s.p, idx.p, idx_s.p, m, 0, end_bit, s));
    heads_kernel<<<grid(m), BS, 0, s>>>(m, keys_s.p, head.p); countLaunch();
    PB_CUDA(cudaMemsetAsync(head.p + m, 0, sizeof(int), s));
    size_t tb2 = 0;
    PB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb2, head.p, mid.p, m + 1, s));
    TmpBuf<unsigned char> tmp2(std::max<size_t>(tb2, 1), s);
    PB_CUDA(cub::DeviceScan::ExclusiveSum(tmp2.p, tb2, head.p, mid.p, m + 1, s));
    int nnz_c = 0;
    PB_CUDA(cudaMemcpyAsync(&nnz_c, mid.p + m, sizeof(int), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
    // restriction data + coarse CSR
    L.gal_seg.alloc(ar, nnz_c + 1, s);
    L.gal_src.alloc(ar, m, s);
    C.n = nc;
    C.nnz = nnz_c;
    C.o_rowptr.alloc(ar, nc + 1, s);
    C.o_col.alloc(ar, nnz_c, s);
    coarse_csr_kernel<<<grid(m), BS, 0, s>>>(m, keys_s.p, head.p, mid.p, idx_s.p, L.csr_pos, nc, L.gal_seg.p,
                                             C.o_col.p, C.o_rowptr.p, L.gal_src.p); countLaunch();
    int hm = (int)m;
    PB_CUDA(cudaMemcpyAsync(L.gal_seg.p + nnz_c, &hm, sizeof(int), cudaMemcpyHostToDevice, s));
    PB_CUDA(cudaMemcpyAsync(C.o_rowptr.p + nc, &nnz_c, sizeof(int), cudaMemcpyHostToDevice, s));
    // coarse SELL
    C.nslices = ceil_div(nc, 32);
    TmpBuf<int> se(C.nslices + 1, s);
    PB_CUDA(cudaMemsetAsync(se.p + C.nslices, 0, sizeof(int), s));
    rowlen_slice_kernel<<<grid(C.nslices), BS, 0, s>>>(nc, C.nslices, C.o_rowptr.p, se.p); countLaunch();
    C.o_sl_off.alloc(ar, C.nslices + 1, s);
    size_t tb3 = 0;
    PB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb3, se.p, C.o_sl_off.p, C.nslices + 1, s));
    TmpBuf<unsigned char> tmp3(std::max<size_t>(tb3, 1), s);
    PB_CUDA(cub::DeviceScan::ExclusiveSum(tmp3.p, tb3, se.p, C.o_sl_off.p, C.nslices + 1, s));
    int sell = 0;
    PB_CUDA(cudaMemcpyAsync(&sell, C.o_sl_off.p + C.nslices, sizeof(int), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
    C.sell_nnz = sell;
    C.o_sl_col.alloc(ar, std::max(sell, 1), s);
    C.o_csr_pos.alloc(ar, std::max(nnz_c, 1), s);
    C.o_diag_pos.alloc(ar, nc, s);
    sell_fill_kernel<<<grid((int64_t)C.nslices * 32), BS, 0, s>>>(nc, C.nslices, C.o_rowptr.p, C.o_col.p,
                                                                   C.o_sl_off.p, C.o_sl_col.p, C.o_csr_pos.p,
                                                                   C.o_diag_pos.p); countLaunch();
    C.rowptr = C.o_rowptr.p;
    C.col = C.o_col.p;
    C.csr_pos = C.o_csr_pos.p;
    C.sl_off = C.o_sl_off.p;
    C.sl_col = C.o_sl_col.p;
    C.diag_pos = C.o_diag_pos.p;
    C.o_vals.alloc(ar, std::max(sell, 1), s);
    C.o_vals.zero(s);
    C.vals = C.o_vals.p;
    PB_LAUNCH("amg galerkin structure");
}

void galerkinValues(const AmgLevel& L, AmgLevel& C, cudaStream_t s) {
    galerkin_values_kernel<<<grid(C.nnz), BS, 0, s>>>((int)C.nnz, L.gal_seg.p, L.gal_src.p, L.vals, C.csr_pos,
                                                       C.o_vals.p); countLaunch();
}

// aggregate -> member rows (rows sorted by aggregate, stable)
void members(DevArena& ar, AmgLevel& L, int nc, cudaStream_t s) {
    const int n = L.n;
    TmpBuf<int> rows(n, s), agg_s(n, s);
    iota_kernel<<<grid(n), BS, 0, s>>>(n, rows.p); countLaunch();
    L.m_idx.alloc(ar, n, s);
    int end_bit = 1;
    while (end_bit < 31 && (1 << end_bit) < nc) ++end_bit;
    size_t tb = 0;
    PB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, L.agg.p, agg_s.p, rows.p, L.m_idx.p, n, 0, end_bit, s));
    TmpBuf<unsigned char> tmp(std::max<size_t>(tb, 1), s);
    PB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, L.agg.p, agg_s.p, rows.p, L.m_idx.p, n, 0, end_bit, s));
    L.m_off.alloc(ar, nc + 1, s);
    member_heads_kernel<<<grid(n), BS, 0, s>>>(n, agg_s.p, L.m_off.p); countLaunch();
    PB_CUDA(cudaMemcpyAsync(L.m_off.p + nc, &n, sizeof(int), cudaMemcpyHostToDevice, s));
    PB_CUDA(cudaStreamSynchronize(s));
    PB_LAUNCH("amg members");
}

// Smoothed restriction Rt of level L (aggregates L.agg, nc of them): the fine
// entries (i, j) sorted by (agg(i), j); each distinct key is one Rt entry.
void restrictionStructure(DevArena& ar, AmgLevel& L, int nc, cudaStream_t s) {
    const int n = L.n;
    const int64_t m = L.nnz;
    TmpBuf<long long> keys(m, s), keys_s(m, s);
    TmpBuf<int> idx(m, s), idx_s(m, s), head(m + 1, s), mid(m + 1, s);
    rt_keys_kernel<<<grid(n), BS, 0, s>>>(n, L.rowptr, L.col, L.agg.p, (long long)n, keys.p, idx.p); countLaunch();
    int end_bit = 1;
    while (end_bit < 63 && ((long long)1 << end_bit) < (long long)nc * n) ++end_bit;
    size_t tb = 0;
    PB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.p, keys_s.p, idx.p, idx_s.p, m, 0, end_bit, s));
    TmpBuf<unsigned char> tmp(std::max<size_t>(tb, 1), s);
    PB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, keys.p, keys_s.p, idx.p, idx_s.p, m, 0, end_bit, s));
    heads_kernel<<<grid(m), BS, 0, s>>>(m, keys_s.p, head.p); countLaunch();
    PB_CUDA(cudaMemsetAsync(head.p + m, 0, sizeof(int), s));
    size_t tb2 = 0;
    PB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb2, head.p, mid.p, m + 1, s));
    TmpBuf<unsigned char> tmp2(std::max<size_t>(tb2, 1), s);
    PB_CUDA(cub::DeviceScan::ExclusiveSum(tmp2.p, tb2, head.p, mid.p, m + 1, s));
    int nnz = 0;
    PB_CUDA(cudaMemcpyAsync(&nnz, mid.p + m, sizeof(int), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
    L.rt_nnz = nnz;
    L.rt_seg.alloc(ar, nnz + 1, s);
    L.rt_src.alloc(ar, m, s);
    L.rt_rowptr.alloc(ar, nc + 1, s);
    L.rt_col.alloc(ar, std::max(nnz, 1), s);
    coarse_csr_kernel<<<grid(m), BS, 0, s>>>(m, keys_s.p, head.p, mid.p, idx_s.p, L.csr_pos, (long long)n,
                                             L.rt_seg.p, L.rt_col.p, L.rt_rowptr.p, L.rt_src.p); countLaunch();
    int hm = (int)m;
    PB_CUDA(cudaMemcpyAsync(L.rt_seg.p + nnz, &hm, sizeof(int), cudaMemcpyHostToDevice, s));
    PB_CUDA(cudaMemcpyAsync(L.rt_rowptr.p + nc, &nnz, sizeof(int), cudaMemcpyHostToDevice, s));
    L.rt_erow.alloc(ar, std::max(nnz, 1), s);
    entry_rows_kernel<<<grid(nc), BS, 0, s>>>(nc, L.rt_rowptr.p, L.rt_erow.p); countLaunch();
    // SELL-C-sigma layout (rows: aggregates, reordered within windows; padded slots
    // point at column 0 with value 0)
    L.rt_nslices = ceil_div(nc, 32);
    {
        TmpBuf<unsigned> keys(nc, s), keys_s(nc, s);
        TmpBuf<int> rows(nc, s);
        L.rt_perm.alloc(ar, std::max(nc, 1), s);
        rt_order_keys_kernel<<<grid(nc), BS, 0, s>>>(nc, L.rt_rowptr.p, keys.p, rows.p); countLaunch();
        int end_bit = 8;
        while (end_bit < 32 && (1u << (end_bit - 8)) <= (unsigned)(nc / RT_SIGMA)) ++end_bit;
        size_t tbo = 0;
        PB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tbo, keys.p, keys_s.p, rows.p, L.rt_perm.p, nc, 0, end_bit, s));
        TmpBuf<unsigned char> tmpo(std::max<size_t>(tbo, 1), s);
        PB_CUDA(cub::DeviceRadixSort::SortPairs(tmpo.p, tbo, keys.p, keys_s.p, rows.p, L.rt_perm.p, nc, 0, end_bit, s));
    }
    TmpBuf<int> se(L.rt_nslices + 1, s);
    PB_CUDA(cudaMemsetAsync(se.p + L.rt_nslices, 0, sizeof(int), s));
    rt_slice_len_kernel<<<grid(L.rt_nslices), BS, 0, s>>>(nc, L.rt_nslices, L.rt_rowptr.p, L.rt_perm.p, se.p); countLaunch();
    L.rt_sl_off.alloc(ar, L.rt_nslices + 1, s);
    size_t tb3 = 0;
    PB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb3, se.p, L.rt_sl_off.p, L.rt_nslices + 1, s));
    TmpBuf<unsigned char> tmp3(std::max<size_t>(tb3, 1), s);
    PB_CUDA(cub::DeviceScan::ExclusiveSum(tmp3.p, tb3, se.p, L.rt_sl_off.p, L.rt_nslices + 1, s));
    int sell = 0;
    PB_CUDA(cudaMemcpyAsync(&sell, L.rt_sl_off.p + L.rt_nslices, sizeof(int), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
    L.rt_sl_col.alloc(ar, std::max(sell, 1), s);
    L.rt_csr_pos.alloc(ar, std::max(nnz, 1), s);
    rt_fill_kernel<<<grid((int64_t)L.rt_nslices * 32), BS, 0, s>>>(nc, L.rt_nslices, L.rt_rowptr.p, L.rt_col.p,
                                                                    L.rt_perm.p, L.rt_sl_off.p, L.rt_sl_col.p,
                                                                    L.rt_csr_pos.p); countLaunch();
    L.rt_vals.alloc(ar, std::max(sell, 1), s);
    L.rt_vals.zero(s);
    L.rt_lpr = lanesPerRow(nc, nnz);
    PB_LAUNCH("amg restriction structure");
}

// returns true if a buffer was allocated
bool allocCycle(DevArena& ar, AmgLevel& L, bool mixed, bool klevel, cudaStream_t s) {
    bool fresh = false;
    int np = L.nslices * 32;
    for (auto* b : {&L.b, &L.x, &L.x2, &L.res, &L.dinv})
        if (!b->p) {
            b->alloc(ar, np, s);
            b->zero(s);
            fresh = true;
        }
    if (klevel)
        for (auto* b : {&L.kz2, &L.kq1, &L.kr1})
            if (!b->p) {
                b->alloc(ar, np, s);
                b->zero(s);
                fresh = true;
            }
    if (mixed) {
        for (auto* b : {&L.b32, &L.x32, &L.x232, &L.res32, &L.dinv32})
            if (!b->p) {
                b->alloc(ar, np, s);
                b->zero(s);
                fresh = true;
            }
        if (!L.vals32.p) {
            L.vals32.alloc(ar, std::max<int64_t>(L.sell_nnz, 1), s);
            L.vals32.zero(s);
            fresh = true;
        }
        if (L.rt_vals.p && !L.rt_vals32.p) {
            L.rt_vals32.alloc(ar, L.rt_vals.n, s);
            L.rt_vals32.zero(s);
            fresh = true;
        }
    }
    return fresh;
}

}  // namespace

namespace {
// process-wide, so a hierarchy's buffers can never match the key of another
// (destroyed) hierarchy that lived at the same address
uint64_t nextGeneration() {
    static std::atomic<uint64_t> g{0};
    return ++g;
}
}  // namespace

void Amg::forPressure() {
    scale = 2.0;
    flex_scale = 2.2;
    const char* e = std::getenv("PRISM_AMG_KCYCLE");
    k_levels = e && e[0] ? std::max(0, std::atoi(e)) : 0;
    k_mask = 0;
    for (int l = 1; l <= k_levels && l < 31; ++l) k_mask |= 1u << l;
    // PRISM_AMG_KLEVELS: the K levels as a list ("2" or "2,3")
    if (const char* m = std::getenv("PRISM_AMG_KLEVELS")) {
        k_mask = 0;
        for (const char* q = m; *q;) {
            const int l = std::atoi(q);
            if (l >= 1 && l < 31) k_mask |= 1u << l;
            while (*q && *q != ',') ++q;
            if (*q == ',') ++q;
        }
        k_levels = 0;
        for (int l = 1; l < 31; ++l)
            if (k_mask >> l & 1u) k_levels = l;
    }
}

bool Amg::kLevel(size_t l) const {
    return l >= 1 && l < 31 && (k_mask >> l & 1u) && l + 1 < levels.size() && (tail < 0 || (int)l < tail);
}

void Amg::setup(const SellMatrix& A, const int* rowptr, const int* col, bool mixed, cudaStream_t s) {
    if (values_current && built && !levels.empty() && levels[0]->n == A.n && levels[0]->sl_off == A.sl_off &&
        levels[0]->vals == A.vals && (!mixed || has32))
        return;
    if (!built || levels.empty() || levels[0]->n != A.n || levels[0]->sl_off != A.sl_off) {
        levels.clear();
        coarse_a.release();
        coarse_inv.release();
        coarse_inv32.release();
        coarse_bad.release();
        kscal.release();
        kpart.release();
        kcount.release();
        arena.reset();  // stream order keeps earlier work on the old hierarchy ahead of its reuse
        auto L0 = std::make_unique<AmgLevel>();
        L0->n = A.n;
        L0->nslices = A.nslices;
        L0->nnz = A.nnz_csr;
        L0->sell_nnz = A.nnz_padded;
        L0->rowptr = rowptr;
        L0->col = col;
        L0->o_csr_pos.alloc(arena, std::max<int64_t>(A.nnz_csr, 1), s);
        csr_pos_kernel<<<grid(A.n), BS, 0, s>>>(A.n, rowptr, A.sl_off, L0->o_csr_pos.p); countLaunch();
        L0->csr_pos = L0->o_csr_pos.p;
        L0->sl_off = A.sl_off;
        L0->sl_col = A.col;
        L0->diag_pos = A.diag_pos;
        L0->vals = A.vals;
        levels.push_back(std::move(L0));
        // PRISM_VERBOSE: host time of the setup phases (stream drained around each)
        double t_match = 0.0, t_gal = 0.0, t_mem = 0.0, t_rt = 0.0;
        auto timed = [&](double& acc, auto&& f) {
            if (!verbose()) return f();
            PB_CUDA(cudaStreamSynchronize(s));
            auto t0 = std::chrono::steady_clock::now();
            auto r = f();
            PB_CUDA(cudaStreamSynchronize(s));
            acc += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            return r;
        };
        while ((int)levels.size() < MAX_LEVELS) {
            AmgLevel& L = *levels.back();
            if (L.n <= COARSE_MAX) break;
            // pass 1
            TmpBuf<int> agg1(L.n, s);
            int n1 = timed(t_match, [&] { return matchPairs(L, agg1.p, s); });
            if (n1 > (int)(0.9 * L.n)) break;
            L.agg.alloc(arena, L.n, s);
            // the pass-1 operator T and the pass-1 restriction data of L are
            // intermediates: their arena space is given back once L.agg is composed
            const DevArena::Mark pass1 = arena.mark();
            AmgLevel T;
            timed(t_gal, [&] {
                galerkinStructure(arena, L, agg1.p, n1, T, s);
                galerkinValues(L, T, s);
                return 0;
            });
            // pass 2 on the pass-1 operator
            TmpBuf<int> agg2(n1, s);
            int n2 = timed(t_match, [&] { return matchPairs(T, agg2.p, s); });
            compose_kernel<<<grid(L.n), BS, 0, s>>>(L.n, agg1.p, agg2.p, L.agg.p); countLaunch();
            arena.rewind(pass1);
            auto C = std::make_unique<AmgLevel>();
            timed(t_gal, [&] {
                galerkinStructure(arena, L, L.agg.p, n2, *C, s);
                galerkinValues(L, *C, s);
                return 0;
            });
            timed(t_mem, [&] {
                members(arena, L, n2, s);
                return 0;
            });

            levels.push_back(std::move(C));
        }
        coarse_n = levels.back()->n;
        for (auto& L : levels) L->lpr = lanesPerRow(L->n, L->nnz);
        tail = -1;
        for (size_t l = 1; l + 1 < levels.size(); ++l)
            if (levels[l]->n <= tailMaxRows() && levels.size() - l <= (size_t)TAIL_MAX_LEVELS) {
                tail = (int)l;
                break;
            }
        // the down-sweep of each level but the coarsest (the fused tail's levels too)
        for (size_t l = 0; l + 1 < levels.size(); ++l) {
            AmgLevel& L = *levels[l];
            L.use_rt = useRestriction(l, L.n, L.nnz);
            if (L.use_rt)
                timed(t_rt, [&] {
                    restrictionStructure(arena, L, levels[l + 1]->n, s);
                    return 0;
                });
        }
        if (verbose()) {
            std::fprintf(stderr, "[prism amg] hierarchy:");
            for (auto& L : levels) std::fprintf(stderr, " %d/%lld/%d", L->n, (long long)L->nnz, L->lpr);
            std::fprintf(stderr, " (rows/entries/lanes per row), coarsest %s, fused tail from level %d; matching %.1f ms, "
                         "galerkin %.1f ms, members %.1f ms, smoothed restriction %.1f ms (levels:",
                         coarse_n <= DENSE_MAX ? "dense" : "Jacobi", tail, t_match, t_gal, t_mem, t_rt);
            for (size_t l = 0; l + 1 < levels.size(); ++l)
                if (levels[l]->use_rt) std::fprintf(stderr, " %zu/%lld", l, (long long)levels[l]->rt_nnz);
            std::fprintf(stderr, ")\n");
        }
        if (coarse_n <= DENSE_MAX) {
            coarse_a.alloc(arena, (size_t)coarse_n * coarse_n, s);
            coarse_inv.alloc(arena, (size_t)coarse_n * coarse_n, s);
            coarse_bad.alloc(arena, 1, s);
            PB_CUDA(cudaFuncSetAttribute(gauss_jordan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         DENSE_MAX * DENSE_MAX * (int)sizeof(double)));
        }
        // smoother weight and coarse-correction factor (PRISM_AMG_OMEGA / PRISM_AMG_SCALE override them)
        if (const char* e = std::getenv("PRISM_AMG_OMEGA")) omega = std::atof(e);
        if (const char* e = std::getenv("PRISM_AMG_SCALE")) scale = std::atof(e);
        if (const char* e = std::getenv("PRISM_AMG_FLEX_SCALE")) flex_scale = std::atof(e);
        built = true;
        generation = nextGeneration();
    } else if (levels[0]->vals != A.vals) {
        levels[0]->vals = A.vals;
        generation = nextGeneration();
    }
    for (size_t l = 0; l < levels.size(); ++l)
        if (allocCycle(arena, *levels[l], mixed, kLevel(l), s)) generation = nextGeneration();
    if (k_levels > 0 && !kscal.p) {
        kscal.alloc(arena, (size_t)KS_N * MAX_LEVELS, s);
        kscal.zero(s);
        kpart.alloc(arena, (size_t)K_MAX_GRID * 4, s);
        kcount.alloc(arena, 1, s);
        kcount.zero(s);
        generation = nextGeneration();
    }
    if (mixed && coarse_inv.p && !coarse_inv32.p) {
        coarse_inv32.alloc(arena, coarse_inv.n, s);
        generation = nextGeneration();
    }
    has32 = mixed;
    // values of every level from the current matrix
    for (size_t l = 0; l + 1 < levels.size(); ++l) galerkinValues(*levels[l], *levels[l + 1], s);
    for (auto& L : levels) {
        dinv_kernel<<<grid(L->n), BS, 0, s>>>(L->n, L->diag_pos, L->vals, L->dinv.p, mixed ? L->dinv32.p : nullptr); countLaunch();
        if (mixed) {
            to_float_kernel<<<std::min<int64_t>(grid(L->sell_nnz), NUM_SMS * 32), BS, 0, s>>>(L->sell_nnz, L->vals,
                                                                                               L->vals32.p); countLaunch();
        }
    }
    for (size_t l = 0; l + 1 < levels.size(); ++l) {
        AmgLevel& L = *levels[l];
        if (!L.use_rt) continue;
        rt_values_kernel<<<grid(L.rt_nnz), BS, 0, s>>>((int)L.rt_nnz, L.rt_erow.p, L.rt_col.p, L.rt_seg.p,
                                                       L.rt_src.p, L.rt_csr_pos.p, L.agg.p, L.vals, L.dinv.p, omega,
                                                       L.rt_vals.p, mixed ? L.rt_vals32.p : nullptr); countLaunch();
    }
    if (verbose() && !capturing(s) && generation != reported_generation) {
        reported_generation = generation;
        std::fprintf(stderr, "[prism amg] hierarchy memory: %.1f MB taken, %.1f MB reserved (fine matrix %.1f MB)\n",
                     arena.used() / 1e6, arena.reserved() / 1e6,
                     (double)levels[0]->sell_nnz * (sizeof(double) + sizeof(int)) / 1e6);
    }
    if (coarse_inv.p) {
        const AmgLevel& C = *levels.back();
        const int n = coarse_n;
        dense_fill_kernel<<<grid(n), BS, 0, s>>>(n, C.rowptr, C.col, C.csr_pos, C.vals, coarse_a.p); countLaunch();
        gauss_jordan_kernel<<<1, 1024, (size_t)n * n * sizeof(double), s>>>(n, coarse_a.p, coarse_inv.p,
                                                                            mixed ? coarse_inv32.p : nullptr,
                                                                            coarse_bad.p); countLaunch();
        if (verbose() && !capturing(s)) {
            int ns = 0;
            PB_CUDA(cudaMemcpyAsync(&ns, coarse_bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
            PB_CUDA(cudaStreamSynchronize(s));
            if (ns) std::fprintf(stderr, "[prism amg] coarsest level: %d singular pivot(s) dropped\n", ns);
        }
    }
    PB_LAUNCH("amg setup");
}

namespace {

template <typename T>
struct CycleData {
    static const T* vals(const AmgLevel& L);
    static const T* rt(const AmgLevel& L);
};
template <>
const double* CycleData<double>::vals(const AmgLevel& L) { return L.vals; }
template <>
const float* CycleData<float>::vals(const AmgLevel& L) { return L.vals32.p; }
template <>
const double* CycleData<double>::rt(const AmgLevel& L) { return L.rt_vals.p; }
template <>
const float* CycleData<float>::rt(const AmgLevel& L) { return L.rt_vals32.p; }

template <typename T>
struct Bufs {
    T *b, *x, *x2, *res;
    const T* dinv;
};
Bufs<double> bufs64(AmgLevel& L) { return {L.b.p, L.x.p, L.x2.p, L.res.p, L.dinv.p}; }
Bufs<float> bufs32(AmgLevel& L) { return {L.b32.p, L.x32.p, L.x232.p, L.res32.p, L.dinv32.p}; }

template <typename T>
bool vcycle(Amg& A, size_t l, const T* b, T* out, const KState* S, cudaStream_t s, bool sample, bool kc,
            const FineProlong<T>* fp = nullptr);

// Whether the coarser level writes level L's xp during its up-sweep (FineProlong). It
// saves two gathers per slot in L's up-sweep and costs the coarser up-sweep one
// scattered write per member: a gain where L's rows are long and a loss on the 2-D
// five-point level 0. Levels with more than 6 entries per row take it, measured on one
// B200: 3-D 128^3 Poisson 91.4 against 95.7 ms (FP64 cycle), 95.0 against 99.0 ms
// (FP32 cycle); 1448^2 cavity SIMPLE 24.34 against 23.94 it/s (23.75 with level 0
// fused too). PRISM_AMG_PROLONG=0 / 1 forces it off / on.
bool prolongFuse(const AmgLevel& L) {
    static const int force = [] {
        const char* e = std::getenv("PRISM_AMG_PROLONG");
        return e && e[0] ? std::atoi(e) : -1;
    }();
    if (force >= 0) return force != 0;
    return L.n > 0 && (double)L.nnz / L.n > 6.0;
}

// K-cycle on level k (FP64): z1 = N.x2 and z2 = N.kz2 from two cycles, the
// combination coefficients in the level's scalars (see k_first_kernel)
void kStep(Amg& A, size_t k, const KState* S, cudaStream_t s) {
    AmgLevel& N = *A.levels[k];
    double* ks = A.kscal.p + (size_t)KS_N * k;
    vcycle<double>(A, k, N.b.p, N.x2.p, S, s, false, true);
    withLpr(N.lpr, [&](auto c) {
        constexpr int P = decltype(c)::value;
        launchPdl(k_first_kernel<P>, kGrid(N.n, P), BS, s, N.n, N.sl_off, N.sl_col, N.vals,
                  (const double*)N.x2.p, (const double*)N.b.p, N.kq1.p, A.kpart.p, A.kcount.p, ks, S);
    });
    launchPdl(k_residual_kernel, grid(N.n), BS, s, N.n, (const double*)N.b.p, (const double*)N.kq1.p,
              (const double*)ks, N.kr1.p, S);
    vcycle<double>(A, k, N.kr1.p, N.kz2.p, S, s, false, true);
    withLpr(N.lpr, [&](auto c) {
        constexpr int P = decltype(c)::value;
        launchPdl(k_second_kernel<P>, kGrid(N.n, P), BS, s, N.n, N.sl_off, N.sl_col, N.vals,
                  (const double*)N.kz2.p, (const double*)N.kq1.p, (const double*)N.kr1.p, A.kpart.p, A.kcount.p,
                  ks, S);
    });
}

// One cycle from level l: out = B b. fp (optional): the finer level's request for its xp
// (FineProlong), written by this level's up-sweep; returns whether it was.
template <typename T>
bool vcycle(Amg& A, size_t l, const T* b, T* out, const KState* S, cudaStream_t s, bool sample, bool kc,
            const FineProlong<T>* fp) {
    AmgLevel& L = *A.levels[l];
    auto B = [&](AmgLevel& X) {
        if constexpr (sizeof(T) == 8) return bufs64(X);
        else return bufs32(X);
    };
    if (A.tail > 0 && (int)l == A.tail) {
        TailParams<T> P{};
        P.nlev = (int)(A.levels.size() - l);
        P.b0 = b;
        if (A.coarse_inv.p) {
            if constexpr (sizeof(T) == 8) P.inv = A.coarse_inv.p;
            else P.inv = A.coarse_inv32.p;
        }
        P.omega = (T)A.omega;
        P.scale = (T)(kc ? A.flex_scale : A.scale);
        P.S = S;
        for (int k = 0; k < P.nlev; ++k) {
            AmgLevel& X = *A.levels[l + k];
            Bufs<T> xb = B(X);
            TailLevel<T>& t = P.L[k];
            t.n = X.n;
            t.nslices = X.nslices;
            t.sl_off = X.sl_off;
            t.col = X.sl_col;
            t.val = CycleData<T>::vals(X);
            t.dinv = xb.dinv;
            t.agg = X.agg.p;
            t.m_off = X.m_off.p;
            t.m_idx = X.m_idx.p;
            t.rt_sl_off = X.rt_sl_off.p;
            t.rt_col = X.rt_sl_col.p;
            t.rt_val = CycleData<T>::rt(X);
            t.rt_perm = X.rt_perm.p;
            t.b = xb.b;
            t.x = xb.x;
            t.x2 = k == 0 ? out : xb.x2;
            t.res = xb.res;
        }
        P.rt = 1;
        for (int k = 0; k + 1 < P.nlev; ++k)
            if (!A.levels[l + k]->use_rt || !P.L[k].rt_val) P.rt = 0;
        launchTail<T>(P, s);
        return false;
    }
    Bufs<T> lb = B(L);
    const T omega = (T)A.omega;
    const T* vals = CycleData<T>::vals(L);
    if (l + 1 == A.levels.size()) {
        if (A.coarse_inv.p) {
            const T* inv;
            if constexpr (sizeof(T) == 8) inv = A.coarse_inv.p;
            else inv = A.coarse_inv32.p;
            launchPdl(coarse_solve_kernel<T>, grid((int64_t)L.n * 32), BS, s, L.n, inv, b, out, S);
        } else {
            // ping-pong between x and res (out is this level's x2 or a caller vector)
            launchPdl(smooth0_kernel<T>, grid(L.n), BS, s, L.n, lb.x, b, lb.dinv, omega, S);
            T* cur = lb.x;
            T* nxt = lb.res;
            for (int k = 0; k < 8; ++k) {
                T* dst = (k == 7) ? out : nxt;
                withLpr(L.lpr, [&](auto c) {
                    constexpr int P = decltype(c)::value;
                    launchPdl(jacobi_sweep_kernel<T, P>, grid((int64_t)L.n * P), BS, s, L.n, L.sl_off, L.sl_col, vals,
                              b, cur, lb.dinv, omega, dst, S);
                });
                nxt = cur;
                cur = dst;
            }
        }
        return false;
    }
    AmgLevel& N = *A.levels[l + 1];
    Bufs<T> nb = B(N);
    const bool fine = sample && l == 0;
    const double mat_bytes = (double)L.nnz * (sizeof(T) + 4) + 4.0 * (L.n + 1);
    const T scale = (T)(kc ? A.flex_scale : A.scale);
    const bool rt = L.use_rt;
    if (rt) {
        // down: bc = Rt b (algorithmic bytes: Rt's entries and columns, its row offsets, b, bc)
        const double rt_bytes =
            (double)L.rt_nnz * (sizeof(T) + 4) + 4.0 * (N.n + 1) + (double)sizeof(T) * (L.n + N.n);
        int slot = fine ? profBegin(PROF_AMG_DOWN, sizeof(T) == 4, rt_bytes, s) : -1;
        withLpr(L.rt_lpr, [&](auto c) {
            constexpr int P = decltype(c)::value;
            auto k = l == 0 ? down_kernel<T, P, true> : down_kernel<T, P, false>;
            launchPdl(k, grid((int64_t)N.n * P), BS, s, N.n, (const int*)L.rt_sl_off.p,
                      (const int*)L.rt_sl_col.p, CycleData<T>::rt(L), (const int*)L.rt_perm.p, b, nb.b, S);
        });
        profEnd(slot, s);
    } else {
        // down: pre-smoothing with the residual (matrix; b, D^-1 read; x, r written), then
        // the members' residuals summed per aggregate
        int slot = fine ? profBegin(PROF_AMG_DOWN, sizeof(T) == 4, mat_bytes + 4.0 * sizeof(T) * L.n, s) : -1;
        withLpr(L.lpr, [&](auto c) {
            constexpr int P = decltype(c)::value;
            launchPdl(pre_kernel<T, P>, grid((int64_t)L.n * P), BS, s, L.n, L.sl_off, L.sl_col, vals, b, lb.dinv,
                      omega, lb.x, lb.res, S);
        });
        profEnd(slot, s);
        launchPdl(restrict_kernel<T>, grid(N.n), BS, s, N.n, (const int*)L.m_off.p, (const int*)L.m_idx.p,
                  (const T*)lb.res, nb.b, S);
    }
    // up: the matrix, b, D^-1 (or x), the aggregate map and out per row, the coarse correction(s)
    const double up_bytes = mat_bytes + ((rt ? 3.0 : 4.0) * sizeof(T) + 4.0) * L.n;
    if constexpr (sizeof(T) == 8) {
        if (kc && A.kLevel(l + 1)) {
            kStep(A, l + 1, S, s);
            const int slot = fine ? profBegin(PROF_AMG_POST, false, up_bytes + 16.0 * N.n, s) : -1;
            withLpr(L.lpr, [&](auto c) {
                constexpr int P = decltype(c)::value;
                auto k = rt ? post_k_kernel<P, false> : post_k_kernel<P, true>;
                launchPdl(k, grid((int64_t)L.n * P), BS, s, L.n, L.sl_off, L.sl_col, vals, b, (const double*)lb.x,
                          (const double*)nb.x2, (const double*)N.kz2.p, (const int*)L.agg.p,
                          (const double*)(A.kscal.p + (size_t)KS_N * (l + 1)), lb.dinv, omega, out, S);
            });
            profEnd(slot, s);
            return false;
        }
    }
    // this level's xp, written by the coarser level's up-sweep into the free res vector
    const FineProlong<T> mine{L.m_off.p, L.m_idx.p, rt ? nullptr : (const T*)lb.x, lb.dinv, b, omega, scale, lb.res};
    const bool have_xp = vcycle<T>(A, l + 1, nb.b, nb.x2, S, s, false, kc, prolongFuse(L) ? &mine : nullptr);
    const FineProlong<T> request = fp ? *fp : FineProlong<T>{};
    const double post_bytes = have_xp ? mat_bytes + 4.0 * sizeof(T) * L.n : up_bytes + (double)sizeof(T) * N.n;
    const int slot = fine ? profBegin(PROF_AMG_POST, sizeof(T) == 4, post_bytes, s) : -1;
    withLpr(L.lpr, [&](auto c) {
        constexpr int P = decltype(c)::value;
        auto k = have_xp ? post_kernel<T, P, 2> : rt ? post_kernel<T, P, 0> : post_kernel<T, P, 1>;
        launchPdl(k, grid((int64_t)L.n * P), BS, s, L.n, L.sl_off, L.sl_col, vals, b, (const T*)lb.x,
                  (const T*)nb.x2, (const int*)L.agg.p, scale, lb.dinv, omega, out, (const T*)lb.res, request, S);
    });
    profEnd(slot, s);
    return fp != nullptr;
}

}  // namespace

void Amg::apply(const double* r, double* z, const KState* S, cudaStream_t s, bool sample) {
    vcycle<double>(*this, 0, r, z, S, s, sample, false);
}
void Amg::apply32(const float* r, float* z, const KState* S, cudaStream_t s, bool flexible, bool sample) {
    vcycle<float>(*this, 0, r, z, S, s, sample, flexible);
}
void Amg::applyK(const double* r, double* z, const KState* S, cudaStream_t s, bool sample) {
    if (k_levels > 0 && !kscal.p) fail(PRISM_INTERNAL, "K-cycle without its buffers (setup first)");
    vcycle<double>(*this, 0, r, z, S, s, sample, true);
}

}  // namespace pb
