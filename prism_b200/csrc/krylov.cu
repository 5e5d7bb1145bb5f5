// krylov.cu -- SELL-32 SpMV and the BiCGSTAB / Jacobi steps of solver::BiCGSTAB
// and solver::Jacobi (numerics/bicgstab.cpp:7-9, numerics/jacobi.cpp:5-9), and
// flexible CG for symmetric systems (the pressure correction; PRISM_SOLVER_FCG).
//
// The reference solves every step() with Eigen's BiCGSTAB + IncompleteLUT to
// machine precision. Here each step runs BiCGSTAB (van der Vorst 1992, the
// textbook recurrences Eigen uses) with Jacobi right preconditioning, applied
// by scaling the columns once per step: A' = A D^-1, x' = D x, so every
// iteration is five streaming kernels and no preconditioner pass:
//   p = r + beta (p - w v)                      vector kernel
//   v = A' p ; r0.v -> alpha                    SpMV + fused dot
//   s = r - alpha v                             vector kernel
//   t = A' s ; t.s, t.t -> w                    SpMV + fused dots
//   x += alpha p + w s ; r = s - w t ; r0.r, r.r -> beta, convergence
// Scalars live in device memory (KState); every reduction is a fixed-order
// two-stage tree (block partials, then the last block to finish reduces them),
// so results are bitwise reproducible run to run. The host launches batches of
// iterations and reads the state once per batch; kernels after convergence
// return immediately, so a batch never changes a converged result.
//
// Mixed precision: the same BiCGSTAB with an FP32 copy of A' and FP32 vectors
// (dot products accumulated in FP64), with reliable updates (Sleijpen and van
// der Vorst 1996): the solution correction is accumulated in FP32 and flushed
// into the FP64 solution whenever the iterated residual has dropped by a factor
// delta (default 0.1) since the last flush; the FP64 true residual b - A'x' then
// replaces the FP32 one and the recurrences continue with the Krylov space kept.
// Convergence is only declared on an FP64 true residual.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <tuple>
#include <unordered_map>

#include "krylov.h"
#include "amg.h"
#include "reduce.cuh"

namespace pb {

namespace {

constexpr int BS = 256;
constexpr int WARPS = BS / 32;
constexpr int MAX_GRID = NUM_SMS * 8;

inline int vecGrid(int n) { return std::max(1, std::min(ceil_div(n, BS), MAX_GRID)); }
inline int spmvGrid(int nslices) { return std::max(1, std::min(ceil_div(nslices, WARPS), NUM_SMS * 16)); }
inline int sliceGrid(int nslices) { return std::max(1, std::min(ceil_div(nslices, WARPS), NUM_SMS * 16)); }

int smCount() {
    static const int c = [] {
        int d = 0, v = 0;
        cudaGetDevice(&d);
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d);
        return v > 0 ? v : NUM_SMS;
    }();
    return c;
}

// Grid of at most one wave of resident blocks: kernels ending in reduceLast()
// pay the per-block publish (fence + atomic) once per block, so a single wave
// keeps that tail off the critical path.
template <typename K>
int waveGrid(K kernel, int needed) {
    static std::mutex mu;
    static std::unordered_map<const void*, int> occ;
    int per_sm = 1;
    {
        std::lock_guard<std::mutex> g(mu);
        auto it = occ.find(reinterpret_cast<const void*>(kernel));
        if (it == occ.end()) {
            int b = 0;
            PB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, BS, 0));
            it = occ.emplace(reinterpret_cast<const void*>(kernel), std::max(b, 1)).first;
        }
        per_sm = it->second;
    }
    return std::max(1, std::min(needed, per_sm * smCount()));
}

// y = A x for a SELL-32 matrix: a warp walks 32-row slices (one row per lane),
// coalesced loads; the matrix is read with evict-first (streaming) loads so
// that L2 keeps the gathered x.
// STAGE 0: plain; 1: alpha = rho / (u.y); 2: w = (u.y)/(y.y)
// The columns and values of up to 8 slots are loaded before their gathers, so
// a row's loads are all in flight at once; the sum runs over the slots in order.
template <typename T, int W = 8, typename TX = T>
__device__ __forceinline__ T sliceRow(const int* __restrict__ col, const T* __restrict__ val,
                                      const TX* __restrict__ x, int b, int width, int lane) {
    T sum = 0;
    for (int j0 = 0; j0 < width; j0 += W) {
        int c[W];
        T v[W];
#pragma unroll
        for (int k = 0; k < W; ++k)
            if (j0 + k < width) {
                c[k] = __ldcs(col + b + 32 * (j0 + k) + lane);
                v[k] = __ldcs(val + b + 32 * (j0 + k) + lane);
            }
#pragma unroll
        for (int k = 0; k < W; ++k)
            if (j0 + k < width) sum += v[k] * (T)__ldg(x + c[k]);
    }
    return sum;
}

template <typename T, int STAGE, int W = 8, int MINB = 5>
__global__ void __launch_bounds__(BS, MINB) spmv_kernel(int nslices, int n, const int* __restrict__ sl_off,
                                                  const int* __restrict__ col, const T* __restrict__ val,
                                                  const T* __restrict__ x, T* __restrict__ y,
                                                  const T* __restrict__ u, double* partials,
                                                  unsigned int* counter, KState* S) {
    pdlEnter();
    if (STAGE != 0 && S->done) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double d0 = 0.0, d1 = 0.0;
    for (int sl = blockIdx.x * WARPS + warp; sl < nslices; sl += gridDim.x * WARPS) {
        const int b = sl_off[sl];
        const int width = (sl_off[sl + 1] - b) >> 5;
        const T sum = sliceRow<T, W>(col, val, x, b, width, lane);
        const int r = sl * 32 + lane;
        y[r] = sum;
        if (STAGE != 0 && r < n) {
            d0 += (double)sum * (double)u[r];
            if (STAGE == 2) d1 += (double)sum * (double)sum;
        }
    }
    if (STAGE == 0) return;
    double v[2] = {d0, d1}, out[2];
    if (reduceLast<2, false>(v, partials, counter, out) && threadIdx.x == 0) {
        if (STAGE == 1) {
            // r0.v = 0 (or a non-finite alpha) breaks the recurrence down: the host restarts
            // from the current x (every later kernel of this iteration returns at once)
            const double alpha = S->rho / out[0];
            if (out[0] == 0.0 || !isfinite(alpha)) S->done = isfinite(out[0]) ? 3 : 5;
            else S->alpha = alpha;
        } else {
            S->ts = out[0];
            S->tt = out[1];
            S->w = out[1] > 0.0 ? out[0] / out[1] : 0.0;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(BS) p_kernel(int n, T* __restrict__ p, const T* __restrict__ r,
                                               const T* __restrict__ v, const KState* S) {
    pdlEnter();
    if (S->done) return;
    const double beta = S->beta, w = S->w;
    for (int i = blockIdx.x * BS + threadIdx.x; i < n; i += gridDim.x * BS)
        p[i] = (T)((double)r[i] + beta * ((double)p[i] - w * (double)v[i]));
}

template <typename T>
__global__ void __launch_bounds__(BS) s_kernel(int n, T* __restrict__ s, const T* __restrict__ r,
                                               const T* __restrict__ v, const KState* S) {
    pdlEnter();
    if (S->done) return;
    const double alpha = S->alpha;
    for (int i = blockIdx.x * BS + threadIdx.x; i < n; i += gridDim.x * BS)
        s[i] = (T)((double)r[i] - alpha * (double)v[i]);
}

// x += alpha p + w q ; r = s - w t  (q = s without a preconditioner pass, else q = M^-1 s, p = M^-1 p)
template <typename T>
__global__ void __launch_bounds__(BS) xr_kernel(int n, T* __restrict__ x, T* __restrict__ r, const T* __restrict__ p,
                                                const T* __restrict__ q, const T* __restrict__ s,
                                                const T* __restrict__ t, const T* __restrict__ r0, double* partials,
                                                unsigned int* counter, KState* S) {
    pdlEnter();
    if (S->done) return;
    const double alpha = S->alpha, w = S->w;
    double d0 = 0.0, d1 = 0.0;
    for (int i = blockIdx.x * BS + threadIdx.x; i < n; i += gridDim.x * BS) {
        double si = (double)s[i];
        double xi = (double)x[i] + alpha * (double)p[i] + w * (double)q[i];
        T ri = (T)(si - w * (double)t[i]);
        x[i] = (T)xi;
        r[i] = ri;
        d0 += (double)r0[i] * (double)ri;
        d1 += (double)ri * (double)ri;
    }
    double v[2] = {d0, d1}, out[2];
    if (reduceLast<2, false>(v, partials, counter, out) && threadIdx.x == 0) {
        S->rr = out[1];
        S->iter += 1;
        const double rho_new = out[0];
        if (!isfinite(out[0]) || !isfinite(out[1])) S->done = 5;
        else if (S->reliable && (out[1] <= S->tol2 || out[1] < S->delta2 * S->rr_update)) S->done = 6;
        else if (out[1] <= S->tol2) S->done = 1;
        else if (S->iter >= S->maxit) S->done = 2;
        else if (w == 0.0 || fabs(rho_new) < EPSILON * EPSILON * S->r0sq) S->done = 3;
        else {
            S->beta = (rho_new / S->rho) * (alpha / w);
            S->rho = rho_new;
        }
    }
}

// r = b - r (r holds A x) or r = b (x = 0); r0 = r; p = v = 0; set up the state.
template <typename T>
__global__ void __launch_bounds__(BS) init_kernel(int n, T* __restrict__ r, const T* __restrict__ b,
                                                  T* __restrict__ r0, T* __restrict__ p, T* __restrict__ v,
                                                  int from_zero, double tol, double* partials,
                                                  unsigned int* counter, KState* S) {
    double d0 = 0.0, d1 = 0.0;
    for (int i = blockIdx.x * BS + threadIdx.x; i < n; i += gridDim.x * BS) {
        double bi = (double)b[i];
        T ri = from_zero ? b[i] : (T)(bi - (double)r[i]);
        r[i] = ri;
        r0[i] = ri;
        p[i] = 0;
        v[i] = 0;
        d0 += (double)ri * (double)ri;
        d1 += bi * bi;
    }
    double vv[2] = {d0, d1}, out[2];
    if (reduceLast<2, false>(vv, partials, counter, out) && threadIdx.x == 0) {
        S->rr = out[0];
        S->bb = out[1];
        S->r0sq = out[0];
        S->tol2 = tol * tol * out[1];
        S->rho = out[0];
        S->beta = out[0];
        S->alpha = 1.0;
        S->w = 1.0;
        if (!isfinite(out[0]) || !isfinite(out[1])) S->done = 5;
        else if (out[1] == 0.0) S->done = 4;
        else if (out[0] <= S->tol2) S->done = 1;
        else S->done = 0;
    }
}

// ---- flexible CG (FP64 recurrences; B one AMG cycle: the FP32 V-cycle, or the FP64
// cycle with K-cycle levels): per iteration
//   z = B r                                          AMG (apply32 / applyK)
//   u = A z ; z.q, z.u, z.r                          SpMV + fused dots
//   beta = (z.q)/dq ; dq' = z.u - beta (z.q) ; dr' = z.r - beta dr ; alpha = dr'/dq'
//   d = z - beta d ; q = u - beta q ; x += alpha d ; r -= alpha q ; r.r, d.q, d.r
// (q = A d is carried, not recomputed: A d = A z - beta A d_prev). dq and dr
// are the previous direction's d.q and d.r, taken exactly in the update pass;
// dq' expands d.q for symmetric A.

// r = b - r (r holds A x); d = q = 0; state as init_kernel
__global__ void __launch_bounds__(BS) fcg_init_kernel(int n, double* __restrict__ r, const double* __restrict__ b,
                                                      double* __restrict__ d, double* __restrict__ q,
                                                      float* __restrict__ r32, double tol, double* partials,
                                                      unsigned int* counter, KState* S) {
    double d0 = 0.0, d1 = 0.0;
    for (int i = blockIdx.x * BS + threadIdx.x; i < n; i += gridDim.x * BS) {
        const double bi = b[i], ri = bi - r[i];
        r[i] = ri;
        if (r32) r32[i] = (float)ri;
        d[i] = 0.0;
        q[i] = 0.0;
        d0 += ri * ri;
        d1 += bi * bi;
    }
    double vv[2] = {d0, d1}, out[2];
    if (reduceLast<2, false>(vv, partials, counter, out) && threadIdx.x == 0) {
        S->rr = out[0];
        S->bb = out[1];
        S->r0sq = out[0];
        S->tol2 = tol * tol * out[1];
        S->dq = 1.0;
        S->dr = 0.0;
        S->alpha = 0.0;
        S->beta = 0.0;
        if (!isfinite(out[0]) || !isfinite(out[1])) S->done = 5;
        else if (out[1] == 0.0) S->done = 4;
        else if (out[0] <= S->tol2) S->done = 1;
        else S->done = 0;
    }
}

// u = A z with the dots z.q, z.u, z.r -> beta, alpha (non-positive d.q: restart);
// z in FP64 or FP32 (the preconditioner's precision)
template <int W, int MINB, typename TZ>
__global__ void __launch_bounds__(BS, MINB) fcg_spmv_kernel(int nslices, int n, const int* __restrict__ sl_off,
                                                      const int* __restrict__ col, const double* __restrict__ val,
                                                      const TZ* __restrict__ z, double* __restrict__ u,
                                                      const double* __restrict__ q, const double* __restrict__ r,
                                                      double* partials, unsigned int* counter, KState* S) {
    pdlEnter();
    if (S->done) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double d0 = 0.0, d1 = 0.0, d2 = 0.0;
    for (int sl = blockIdx.x * WARPS + warp; sl < nslices; sl += gridDim.x * WARPS) {
        const int b = sl_off[sl];
        const int width = (sl_off[sl + 1] - b) >> 5;
        const double sum = sliceRow<double, W, TZ>(col, val, z, b, width, lane);
        const int i = sl * 32 + lane;
        u[i] = sum;
        if (i < n) {
            const double zi = (double)z[i];
            d0 += zi * q[i];
            d1 += zi * sum;
            d2 += zi * r[i];
        }
    }
    double v[3] = {d0, d1, d2}, out[3];
    if (reduceLast<3, false>(v, partials, counter, out) && threadIdx.x == 0) {
        const double beta = out[0] / S->dq;
        const double dq = out[1] - beta * out[0];
        const double dr = out[2] - beta * S->dr;
        const double alpha = dr / dq;
        if (!isfinite(out[0]) || !isfinite(out[1]) || !isfinite(out[2])) S->done = 5;
        else if (!(dq > 0.0) || !isfinite(alpha)) S->done = 3;
        else {
            S->beta = beta;
            S->alpha = alpha;
        }
    }
}

// d = z - beta d ; q = u - beta q ; x += alpha d ; r -= alpha q ; r.r, d.q, d.r -> convergence
// (r32: the FP32 copy of r that an FP32 preconditioner reads)
template <typename TZ>
__global__ void __launch_bounds__(BS) fcg_update_kernel(int n, double* __restrict__ x, double* __restrict__ r,
                                                        double* __restrict__ d, double* __restrict__ q,
                                                        const TZ* __restrict__ z, const double* __restrict__ u,
                                                        float* __restrict__ r32, double* partials,
                                                        unsigned int* counter, KState* S) {
    pdlEnter();
    if (S->done) return;
    const double alpha = S->alpha, beta = S->beta;
    double d0 = 0.0, d1 = 0.0, d2 = 0.0;
    for (int i = blockIdx.x * BS + threadIdx.x; i < n; i += gridDim.x * BS) {
        const double di = (double)z[i] - beta * d[i];
        const double qi = u[i] - beta * q[i];
        const double ri = r[i] - alpha * qi;
        x[i] += alpha * di;
        d[i] = di;
        q[i] = qi;
        r[i] = ri;
        if (r32) r32[i] = (float)ri;
        d0 += ri * ri;
        d1 += di * qi;
        d2 += di * ri;
    }
    double v[3] = {d0, d1, d2}, out[3];
    if (reduceLast<3, false>(v, partials, counter, out) && threadIdx.x == 0) {
        S->rr = out[0];
        S->dq = out[1];
        S->dr = out[2];
        S->iter += 1;
        if (!isfinite(out[0]) || !isfinite(out[1])) S->done = 5;
        else if (out[0] <= S->tol2) S->done = 1;
        else if (S->iter >= S->maxit) S->done = 2;
        else if (!(out[1] > 0.0)) S->done = 3;
    }
}

// column scaling: dinv = 1/diag (1 where diag == 0), As = A dinv[col], xs = diag x
__global__ void dinv_kernel(int n, const int* diag_pos, const double* vals, double* dinv, const double* x, double* xs) {
    int i = blockIdx.x * BS + threadIdx.x;
    if (i >= n) return;
    double d = vals[diag_pos[i]];
    double di = (d != 0.0) ? 1.0 / d : 1.0;
    dinv[i] = di;
    if (xs) xs[i] = (d != 0.0) ? d * x[i] : x[i];
}
template <typename T>
__global__ void scale_kernel(int64_t nnz, const int* col, const double* vals, const double* dinv, T* out) {
    for (int64_t k = blockIdx.x * (int64_t)BS + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * BS)
        out[k] = (T)(vals[k] * dinv[col[k]]);
}
__global__ void unscale_kernel(int n, const double* dinv, const double* xs, double* x) {
    int i = blockIdx.x * BS + threadIdx.x;
    if (i < n) x[i] = dinv[i] * xs[i];
}
// refinement: r = b - A x (FP64) -> r (double) and r32; dots r.r, b.b
__global__ void __launch_bounds__(BS) refine_residual_kernel(int n, const double* __restrict__ Ax,
                                                             const double* __restrict__ b, float* __restrict__ r32,
                                                             double* partials, unsigned int* counter, double* out2) {
    double d0 = 0.0, d1 = 0.0;
    for (int i = blockIdx.x * BS + threadIdx.x; i < n; i += gridDim.x * BS) {
        double ri = b[i] - Ax[i];
        r32[i] = (float)ri;
        d0 += ri * ri;
        d1 += b[i] * b[i];
    }
    double v[2] = {d0, d1}, out[2];
    if (reduceLast<2, false>(v, partials, counter, out) && threadIdx.x == 0) {
        out2[0] = out[0];
        out2[1] = out[1];
    }
}
__global__ void fill_zero_f(int n, float* x) {
    int i = blockIdx.x * BS + threadIdx.x;
    if (i < n) x[i] = 0.0f;
}

// Reliable update, part 1: xs += y (FP32 correction flushed into the FP64 solution), y = 0.
__global__ void flush_kernel(int n, double* __restrict__ xs, float* __restrict__ y) {
    int i = blockIdx.x * BS + threadIdx.x;
    if (i < n) {
        xs[i] += (double)y[i];
        y[i] = 0.0f;
    }
}
// Reliable update, part 2 (Ax = A' xs already in `ax`): r64 = b - ax, r32 = (float) r64,
// rr = r64.r64, rho = r0.r32; continue the recurrence or declare convergence.
// first != 0: (re)start -- r0 = r32, p = v = 0, fresh recurrence scalars.
__global__ void __launch_bounds__(BS) reliable_kernel(int n, const double* __restrict__ ax, const double* __restrict__ b,
                                                      double* __restrict__ r64, float* __restrict__ r32,
                                                      float* __restrict__ r032, float* __restrict__ p32,
                                                      float* __restrict__ v32, int first, double tol,
                                                      double* partials, unsigned int* counter, KState* S) {
    double d0 = 0.0, d1 = 0.0, d2 = 0.0;
    for (int i = blockIdx.x * BS + threadIdx.x; i < n; i += gridDim.x * BS) {
        double ri = b[i] - ax[i];
        float rf = (float)ri;
        r64[i] = ri;
        r32[i] = rf;
        if (first) {
            r032[i] = rf;
            p32[i] = 0.0f;
            v32[i] = 0.0f;
        }
        d0 += ri * ri;
        d1 += (double)(first ? rf : r032[i]) * (double)rf;
        d2 += b[i] * b[i];
    }
    double v[3] = {d0, d1, d2}, out[3];
    if (reduceLast<3, false>(v, partials, counter, out) && threadIdx.x == 0) {
        S->rr = out[0];
        S->rr_update = out[0];
        if (first) {
            S->bb = out[2];
            S->tol2 = tol * tol * out[2];
            S->r0sq = out[1];
            S->rho = out[1];
            S->beta = out[1];
            S->alpha = 1.0;
            S->w = 1.0;
        }
        if (!isfinite(out[0]) || !isfinite(out[1])) S->done = 5;
        else if (out[2] == 0.0) S->done = 4;
        else if (out[0] <= S->tol2) S->done = 1;
        else if (S->iter >= S->maxit) S->done = 2;
        else {
            if (!first) {
                if (S->w == 0.0 || fabs(out[1]) < EPSILON * EPSILON * S->r0sq) {
                    S->done = 3;
                    return;
                }
                S->beta = (out[1] / S->rho) * (S->alpha / S->w);
                S->rho = out[1];
            }
            S->done = 0;
        }
    }
}

// Jacobi: out = x + dinv (b - A x)
__global__ void __launch_bounds__(BS) jacobi_kernel(int nslices, int n, const int* __restrict__ sl_off,
                                                    const int* __restrict__ col, const double* __restrict__ val,
                                                    const int* __restrict__ diag_pos, const double* __restrict__ b,
                                                    const double* __restrict__ x, double* __restrict__ out) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int sl = blockIdx.x * WARPS + warp; sl < nslices; sl += gridDim.x * WARPS) {
        const int bo = sl_off[sl], width = (sl_off[sl + 1] - bo) >> 5;
        const int r = sl * 32 + lane;
        if (r >= n) continue;
        double sum = 0.0;
        for (int j = 0; j < width; ++j) sum += val[bo + 32 * j + lane] * x[col[bo + 32 * j + lane]];
        double dinv = 1.0 / val[diag_pos[r]];
        double res = b[r] - sum;
        out[r] = x[r] + dinv * res;
    }
}

// explicit momentum: out = (-(A x - diag x) + b) / diag
__global__ void __launch_bounds__(BS) explicit_kernel(int nslices, int n, const int* __restrict__ sl_off,
                                                      const int* __restrict__ col, const double* __restrict__ val,
                                                      const int* __restrict__ diag_pos, const double* __restrict__ b,
                                                      const double* __restrict__ x, double* __restrict__ out) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int sl = blockIdx.x * WARPS + warp; sl < nslices; sl += gridDim.x * WARPS) {
        const int bo = sl_off[sl], width = (sl_off[sl + 1] - bo) >> 5;
        const int r = sl * 32 + lane;
        if (r >= n) continue;
        double sum = 0.0;
        for (int j = 0; j < width; ++j) sum += val[bo + 32 * j + lane] * x[col[bo + 32 * j + lane]];
        double ac = val[diag_pos[r]];
        double H = sum - ac * x[r];
        out[r] = (-H + b[r]) / ac;
    }
}

// scaled residual pieces: max|Ax - b|, max|diag x|, count of non-finite terms
__global__ void __launch_bounds__(BS) resid_kernel(int nslices, int n, const int* __restrict__ sl_off,
                                                   const int* __restrict__ col, const double* __restrict__ val,
                                                   const int* __restrict__ diag_pos, const double* __restrict__ b,
                                                   const double* __restrict__ x, double* partials,
                                                   unsigned int* counter, double* out3) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double m0 = 0.0, m1 = 0.0, bad = 0.0;
    for (int sl = blockIdx.x * WARPS + warp; sl < nslices; sl += gridDim.x * WARPS) {
        const int bo = sl_off[sl], width = (sl_off[sl + 1] - bo) >> 5;
        const int r = sl * 32 + lane;
        if (r >= n) continue;
        double sum = 0.0;
        for (int j = 0; j < width; ++j) sum += val[bo + 32 * j + lane] * x[col[bo + 32 * j + lane]];
        double e = fabs(sum - b[r]);
        double d = fabs(val[diag_pos[r]] * x[r]);
        if (!isfinite(e) || !isfinite(d)) bad = 1.0;
        else {
            m0 = fmax(m0, e);
            m1 = fmax(m1, d);
        }
    }
    double v[3] = {m0, m1, bad}, out[3];
    if (reduceLast<3, true>(v, partials, counter, out) && threadIdx.x == 0) {
        out3[0] = out[0];
        out3[1] = out[1];
        out3[2] = out[2];
    }
}

// max over rows of sum_{j != i} |a_ij| / |a_ii| (infinite for a zero or non-finite diagonal)
__global__ void __launch_bounds__(BS) offdiag_ratio_kernel(int nslices, int n, const int* __restrict__ sl_off,
                                                           const int* __restrict__ col, const double* __restrict__ val,
                                                           double* partials, unsigned int* counter, double* out1) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double m = 0.0;
    for (int sl = blockIdx.x * WARPS + warp; sl < nslices; sl += gridDim.x * WARPS) {
        const int bo = sl_off[sl], width = (sl_off[sl + 1] - bo) >> 5;
        const int r = sl * 32 + lane;
        if (r >= n) continue;
        double off = 0.0, diag = 0.0;
        for (int j = 0; j < width; ++j) {
            const double a = fabs(val[bo + 32 * j + lane]);
            if (col[bo + 32 * j + lane] == r) diag += a;
            else off += a;
        }
        const double t = off / diag;
        m = (diag > 0.0 && isfinite(t)) ? fmax(m, t) : INFINITY;
    }
    double v[1] = {m}, out[1];
    if (reduceLast<1, true>(v, partials, counter, out) && threadIdx.x == 0) out1[0] = out[0];
}

}  // namespace

// Fresh buffers are zeroed with cudaMemset on the legacy stream, then that
// stream is drained so the zeros land before any kernel of the (non-blocking)
// solve stream reads them.
void KrylovWork::ensure(int n_pad, int64_t nnz_padded, bool mixed) {
    if (!host_state) PB_CUDA(cudaMallocHost(&host_state, sizeof(KState) + 64));
    bool fresh = false;
    if (n != n_pad || nnz != nnz_padded) {
        fresh = true;
        n = n_pad;
        nnz = nnz_padded;
        for (auto* b : {&r, &r0, &p, &v, &s, &t, &xs, &dinv, &tmp}) b->alloc(n_pad);
        As.alloc(nnz_padded);
        partials.alloc((size_t)std::max(ceil_div(n_pad / 32, WARPS), std::max(NUM_SMS, smCount()) * 16) * 4);
        counter.alloc(1);
        PB_CUDA(cudaMemset(counter.p, 0, sizeof(unsigned int)));
        scal.alloc(8);
        state.alloc(1);
        As32.release();
        for (auto* b : {&r32, &r032, &p32, &v32, &s32, &t32, &x32}) b->release();
        // zero vectors once so padded rows stay 0
        for (auto* b : {&r, &r0, &p, &v, &s, &t, &xs, &dinv, &tmp}) PB_CUDA(cudaMemset(b->p, 0, n_pad * sizeof(double)));
    }
    if (mixed && !As32) {
        fresh = true;
        As32.alloc(nnz_padded);
        r64.alloc(n_pad);
        PB_CUDA(cudaMemset(r64.p, 0, n_pad * sizeof(double)));
        for (auto* b : {&r32, &r032, &p32, &v32, &s32, &t32, &x32}) {
            b->alloc(n_pad);
            PB_CUDA(cudaMemset(b->p, 0, n_pad * sizeof(float)));
        }
    }
    if (fresh) PB_CUDA(cudaStreamSynchronize(nullptr));
}
void KrylovWork::ensurePrec(bool mixed) {
    bool fresh = false;
    if (y.n != (size_t)n) {
        fresh = true;
        y.alloc(n);
        z.alloc(n);
        PB_CUDA(cudaMemset(y.p, 0, n * sizeof(double)));
        PB_CUDA(cudaMemset(z.p, 0, n * sizeof(double)));
        y32.release();
        z32.release();
    }
    if (mixed && !y32) {
        fresh = true;
        y32.alloc(n);
        z32.alloc(n);
        PB_CUDA(cudaMemset(y32.p, 0, n * sizeof(float)));
        PB_CUDA(cudaMemset(z32.p, 0, n * sizeof(float)));
    }
    if (fresh) PB_CUDA(cudaStreamSynchronize(nullptr));
}
KrylovWork::~KrylovWork() {
    for (auto& g : graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    if (host_state) cudaFreeHost(host_state);
}

void spmv(const SellMatrix& A, const double* x, double* y, cudaStream_t s) {
    spmv_kernel<double, 0><<<sliceGrid(A.nslices), BS, 0, s>>>(A.nslices, A.n, A.sl_off, A.col, A.vals, x, y, nullptr,
                                                              nullptr, nullptr, nullptr); countLaunch();
    PB_LAUNCH("spmv_kernel");
}

namespace {

// ---- sampled kernel timing (prism_profile_start / prism_profile_stop)
struct Sample {
    cudaEvent_t a, b;
    int kind;
    bool fp32;
    double bytes;
    bool closed;
};
struct Profiler {
    bool on = false;
    long long launches0 = 0;
    long long graphs0 = 0;
    int max_samples = 0;
    std::vector<Sample> samples;
    std::vector<cudaEvent_t> pool;
    cudaEvent_t get() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e;
        PB_CUDA(cudaEventCreate(&e));
        return e;
    }
} g_prof;

template <typename T>
double spmvBytes(const SellMatrix& A) {
    return (double)A.nnz_csr * (sizeof(T) + 4) + 4.0 * (A.n + 1) + 2.0 * A.n * sizeof(T);
}
// flexible CG's u = A z: FP64 matrix, z of zbytes, u written, q and r read for the dots
double fcgSpmvBytes(const SellMatrix& A, int zbytes) {
    return (double)A.nnz_csr * 12.0 + 4.0 * (A.n + 1) + (zbytes + 24.0) * A.n;
}

template <typename T>
struct Vecs {
    T *x, *r, *r0, *p, *v, *s, *t;
};

// PRISM_VERBOSE: device time of a scope on stream s, printed to stderr at its end
struct VerboseTimer {
    const char* what;
    cudaStream_t s;
    cudaEvent_t a = nullptr, b = nullptr;
    VerboseTimer(const char* w, cudaStream_t st) : what(w), s(st) {
        if (!verbose()) return;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, s);
    }
    ~VerboseTimer() {
        if (!a) return;
        float ms = 0.f;
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        cudaEventElapsedTime(&ms, a, b);
        std::fprintf(stderr, "[prism] %s: %.3f ms\n", what, ms);
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
};

// z = M^-1 r by one AMG V-cycle (FP64 or FP32 hierarchy)
inline void precApply(Amg* amg, const double* r, double* z, const KState* S, cudaStream_t s, bool sample) {
    amg->apply(r, z, S, s, sample);
}
inline void precApply(Amg* amg, const float* r, float* z, const KState* S, cudaStream_t s, bool) {
    amg->apply32(r, z, S, s);
}

// `count` BiCGSTAB iterations on the operator M (SELL values), launched one
// kernel at a time. With amg: right-preconditioned, y = M^-1 p and z = M^-1 s.
// launch shape of the reducing SpMV stages: W slots loaded ahead per lane, at least MINB
// blocks per SM. Measured on the 128^3 transport matrix (ncu, FP64): 4x6 (40 registers,
// 71% warps active) 45 / 43 us for the two stages against 47 / 53 us for 8x5 (48
// registers, 60%) and 52 / 50 us for 4x8 (32 registers, 97%). PRISM_SPMV_SHAPE = "WxMINB"
// (4x6, 8x5, 4x8) overrides it.
int spmvShape() {
    static const int v = [] {
        const char* e = std::getenv("PRISM_SPMV_SHAPE");
        if (!e || !e[0]) return 3;
        const std::string t(e);
        return t == "4x8" ? 1 : t == "8x5" ? 0 : 3;
    }();
    return v;
}
template <typename T, int STAGE, typename F>
void withSpmvShape(F&& f) {
    switch (spmvShape()) {
        case 0: f(spmv_kernel<T, STAGE, 8, 5>); break;
        case 1: f(spmv_kernel<T, STAGE, 4, 8>); break;
        default: f(spmv_kernel<T, STAGE, 4, 6>); break;
    }
}

template <typename T>
void iterateEager(const SellMatrix& A, const T* M, Vecs<T> V, Amg* amg, T* y, T* z, long long count, bool sample,
                  KrylovWork& w, cudaStream_t s) {
    KState* S = w.state.p;
    const int n = A.n, vg = vecGrid(n);
    decltype(&spmv_kernel<T, 1>) k1 = nullptr;
    decltype(&spmv_kernel<T, 2>) k2 = nullptr;
    withSpmvShape<T, 1>([&](auto k) { k1 = k; });
    withSpmvShape<T, 2>([&](auto k) { k2 = k; });
    const int sg1 = waveGrid(k1, ceil_div(A.nslices, WARPS));
    const int sg2 = waveGrid(k2, ceil_div(A.nslices, WARPS));
    for (long long it = 0; it < count; ++it) {
        launchPdl(p_kernel<T>, vg, BS, s, n, V.p, V.r, V.v, S);
        const T* dp = V.p;
        if (amg) {
            precApply(amg, V.p, y, S, s, sample);
            dp = y;
        }
        const int slot = sample ? profBegin(PROF_SPMV, sizeof(T) == 4, spmvBytes<T>(A), s) : -1;
        launchPdl(k1, sg1, BS, s, A.nslices, n, A.sl_off, A.col, M, dp, V.v, V.r0, w.partials.p,
                  w.counter.p, S);
        profEnd(slot, s);
        launchPdl(s_kernel<T>, vg, BS, s, n, V.s, V.r, V.v, S);
        const T* ds = V.s;
        if (amg) {
            precApply(amg, V.s, z, S, s, sample);
            ds = z;
        }
        launchPdl(k2, sg2, BS, s, A.nslices, n, A.sl_off, A.col, M, ds, V.t, V.s, w.partials.p,
                  w.counter.p, S);
        launchPdl(xr_kernel<T>, vg, BS, s, n, V.x, V.r, dp, ds, V.s, V.t, V.r0, w.partials.p, w.counter.p, S);
    }
}

// Krylov method of a solve: BiCGSTAB, or flexible CG preconditioned by an FP64
// cycle (with the K-cycle levels) or by an FP32 V-cycle
enum { KM_BICGSTAB = 0, KM_FCG = 1, KM_FCG_PRE32 = 2 };

// `count` flexible-CG iterations (FP64 recurrences), launched one kernel at a time.
// Vectors: x = V.x, r = V.r, d = V.p, q = V.v, u = V.t; z = y (KM_FCG) or, for
// KM_FCG_PRE32, the FP32 pair r32 = w.y32 -> z32 = w.z32.
void iterateFcgEager(const SellMatrix& A, const double* M, Vecs<double> V, Amg* amg, double* y, int mode,
                     long long count, bool sample, KrylovWork& w, cudaStream_t s) {
    KState* S = w.state.p;
    const int n = A.n, vg = vecGrid(n);
    const bool p32 = mode == KM_FCG_PRE32;
    auto k64 = fcg_spmv_kernel<4, 6, double>;
    auto k32 = fcg_spmv_kernel<4, 6, float>;
    const int sg = p32 ? waveGrid(k32, ceil_div(A.nslices, WARPS)) : waveGrid(k64, ceil_div(A.nslices, WARPS));
    for (long long it = 0; it < count; ++it) {
        if (p32) {
            amg->apply32(w.y32.p, w.z32.p, S, s, true, sample);
            const int slot = sample ? profBegin(PROF_FCG_SPMV, false, fcgSpmvBytes(A, 4), s) : -1;
            launchPdl(k32, sg, BS, s, A.nslices, n, A.sl_off, A.col, M, (const float*)w.z32.p, V.t,
                      (const double*)V.v, (const double*)V.r, w.partials.p, w.counter.p, S);
            profEnd(slot, s);
            launchPdl(fcg_update_kernel<float>, vg, BS, s, n, V.x, V.r, V.p, V.v, (const float*)w.z32.p,
                      (const double*)V.t, w.y32.p, w.partials.p, w.counter.p, S);
        } else {
            amg->applyK(V.r, y, S, s, sample);
            const int slot = sample ? profBegin(PROF_FCG_SPMV, false, fcgSpmvBytes(A, 8), s) : -1;
            launchPdl(k64, sg, BS, s, A.nslices, n, A.sl_off, A.col, M, (const double*)y, V.t, (const double*)V.v,
                      (const double*)V.r, w.partials.p, w.counter.p, S);
            profEnd(slot, s);
            launchPdl(fcg_update_kernel<double>, vg, BS, s, n, V.x, V.r, V.p, V.v, (const double*)y,
                      (const double*)V.t, (float*)nullptr, w.partials.p, w.counter.p, S);
        }
    }
}

// PRISM_NO_GRAPHS=1: launch every iteration kernel by kernel (diagnostics)
bool graphsEnabled() {
    static const bool on = [] {
        const char* e = std::getenv("PRISM_NO_GRAPHS");
        return !(e && e[0] && e[0] != '0');
    }();
    return on;
}

// A batch of iterations. The first batch of a solve runs kernel by kernel (and
// feeds the SpMV timing samples); later batches replay one iteration captured
// as a CUDA graph (~90 kernels with an AMG V-cycle on each side), re-captured
// only when an operand changes. Kernels after convergence return at once, so
// replays past the end of a batch change nothing.
template <typename T>
void iterateAny(const SellMatrix& A, const T* M, Vecs<T> V, Amg* amg, T* y, T* z, long long count, bool sample,
                int mode, KrylovWork& w, cudaStream_t s) {
    if constexpr (sizeof(T) == 8) {
        if (mode != KM_BICGSTAB) {
            iterateFcgEager(A, M, V, amg, y, mode, count, sample, w, s);
            return;
        }
    }
    iterateEager<T>(A, M, V, amg, y, z, count, sample, w, s);
}

template <typename T>
void iterate(const SellMatrix& A, const T* M, Vecs<T> V, Amg* amg, T* y, T* z, long long batch, bool first,
             KrylovWork& w, cudaStream_t s, int mode = KM_BICGSTAB) {
    if (first || !graphsEnabled()) {
        iterateAny<T>(A, M, V, amg, y, z, batch, true, mode, w, s);
        return;
    }
    std::vector<uintptr_t> key = {(uintptr_t)mode, (uintptr_t)sizeof(T), (uintptr_t)A.sl_off, (uintptr_t)A.col, (uintptr_t)A.nslices,
                                  (uintptr_t)A.n, (uintptr_t)M, (uintptr_t)V.x, (uintptr_t)V.r, (uintptr_t)V.r0,
                                  (uintptr_t)V.p, (uintptr_t)V.v, (uintptr_t)V.s, (uintptr_t)V.t, (uintptr_t)amg,
                                  (uintptr_t)(amg ? amg->generation : 0), (uintptr_t)y, (uintptr_t)z,
                                  (uintptr_t)w.state.p, (uintptr_t)w.partials.p, (uintptr_t)w.counter.p,
                                  (uintptr_t)w.y32.p, (uintptr_t)w.z32.p};
    constexpr size_t MAX_GRAPHS = 8;
    auto hit = std::find_if(w.graphs.begin(), w.graphs.end(), [&](const KrylovWork::IterGraph& g) { return g.key == key; });
    if (hit != w.graphs.end()) {
        std::rotate(hit, hit + 1, w.graphs.end());  // most recently used last
    } else {
        if (w.graphs.size() >= MAX_GRAPHS) {
            cudaGraphExecDestroy(w.graphs.front().exec);
            w.graphs.erase(w.graphs.begin());
        }
        KrylovWork::IterGraph ng;
        const long long c0 = launchCounter().load();
        const auto t_cap = std::chrono::steady_clock::now();
        PB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        cudaGraph_t graph = nullptr;
        try {
            iterateAny<T>(A, M, V, amg, y, z, 1, false, mode, w, s);
        } catch (...) {
            cudaStreamEndCapture(s, &graph);
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            throw;
        }
        cudaError_t e = cudaStreamEndCapture(s, &graph);
        const long long k = launchCounter().load() - c0;
        launchCounter().fetch_sub(k);
        PB_CUDA(e);
        e = cudaGraphInstantiate(&ng.exec, graph, 0);
        cudaGraphDestroy(graph);
        PB_CUDA(e);
        ng.key = std::move(key);
        ng.kernels = k;
        w.graphs.push_back(std::move(ng));
        if (verbose())
            std::fprintf(stderr, "[prism] iteration graph captured: %lld kernels, %.3f ms\n", k,
                         std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_cap).count());
    }
    const KrylovWork::IterGraph& g = w.graphs.back();
    for (long long it = 0; it < batch; ++it) PB_CUDA(cudaGraphLaunch(g.exec, s));
    launchCounter().fetch_add(g.kernels * batch);
}

// BiCGSTAB iterations on (M, rhs) from the current x; returns iterations done.
template <typename T>
KrylovOut runBicgstab(const SellMatrix& A, const T* M, const T* rhs, Vecs<T> V, bool from_zero, double tol,
                      long long maxit, KrylovWork& w, cudaStream_t s, Amg* amg, T* y, T* z,
                      int mode = KM_BICGSTAB) {
    const bool flex = mode != KM_BICGSTAB;
    KrylovOut out;
    KState* S = w.state.p;
    KState init{};
    init.maxit = maxit;
    PB_CUDA(cudaMemcpyAsync(S, &init, sizeof(KState), cudaMemcpyHostToDevice, s));
    const int n = A.n, vg = vecGrid(n), sg = sliceGrid(A.nslices);
    int restarts = 0;
    bool zero = from_zero;
    long long batch = 8;
    while (true) {
        if (!zero)
            spmv_kernel<T, 0><<<sg, BS, 0, s>>>(A.nslices, n, A.sl_off, A.col, M, V.x, V.r, nullptr, nullptr, nullptr,
                                                nullptr); countLaunch();
        if constexpr (sizeof(T) == 8) {
            if (flex) {
                if (zero) fail(PRISM_INTERNAL, "flexible CG starts from A x");
                fcg_init_kernel<<<vg, BS, 0, s>>>(n, V.r, rhs, V.p, V.v, mode == KM_FCG_PRE32 ? w.y32.p : nullptr, tol,
                                                  w.partials.p, w.counter.p, S); countLaunch();
            }
        }
        if (!flex) {
            init_kernel<T><<<vg, BS, 0, s>>>(n, V.r, rhs, V.r0, V.p, V.v, zero ? 1 : 0, tol, w.partials.p, w.counter.p,
                                             S); countLaunch();
        }
        PB_LAUNCH("bicgstab init");
        zero = false;
        int done = 0;
        bool first = true;
        while (true) {
            iterate<T>(A, M, V, amg, y, z, batch, first, w, s, mode);
            first = false;
            PB_LAUNCH("bicgstab iteration");
            PB_CUDA(cudaMemcpyAsync(w.host_state, S, sizeof(KState), cudaMemcpyDeviceToHost, s));
            PB_CUDA(cudaStreamSynchronize(s));
            done = w.host_state->done;
            if (done != 0) break;
            batch = std::min<long long>(batch * 2, 64);
        }
        out.iterations = w.host_state->iter;
        if (done == 3) {
            if (++restarts > 20) {
                out.status = PRISM_BREAKDOWN;
                break;
            }
            continue;  // restart from the current x (r recomputed from b - A x)
        }
        if (done == 2) out.status = PRISM_NOT_CONVERGED;
        if (done == 5) out.status = PRISM_NONFINITE;
        break;
    }
    return out;
}

}  // namespace

// Mixed precision: the FP32 recurrence restarts from the FP64 solution at every reliable
// update (r0 = the true residual, fresh directions), which measured fewer iterations than
// continuing it (128^2 Poisson with Jacobi: 364 against 662; 128^3 transport with AMG: 124
// against 132) -- continuing it also stalled for 14,000 iterations on the Poisson problem.
// PRISM_MIXED_RESTART=0 continues it instead. Either way a segment longer than kStallFactor
// x the longest earlier one (and than kStallMin iterations) is restarted.
constexpr long long kStallMin = 64, kStallFactor = 8;
bool restartOnUpdate() {
    static const bool v = [] {
        const char* e = std::getenv("PRISM_MIXED_RESTART");
        return !(e && e[0] == '0');
    }();
    return v;
}

namespace {
// flexible CG's preconditioner: an FP32 V-cycle (half the bytes of the FP64 one; the
// recurrences stay FP64) unless the hierarchy has K-cycle levels (FP64 only) or
// PRISM_FCG_PREC=fp64
int fcgMode(const Amg* amg) { return fcgPre32(amg) ? KM_FCG_PRE32 : KM_FCG; }
}  // namespace

bool fcgPre32(const Amg* amg) {
    static const bool p64 = [] {
        const char* e = std::getenv("PRISM_FCG_PREC");
        return e && std::strcmp(e, "fp64") == 0;
    }();
    return !p64 && amg->k_levels == 0;
}

KrylovOut bicgstab(const SellMatrix& A, const double* b, double* x, double tol, long long maxit, int precision,
                   double inner_tol, KrylovWork& w, cudaStream_t s, Amg* amg, const int* rowptr, const int* col,
                   bool flexible) {
    const bool mixed = precision == PRISM_PREC_MIXED;
    if (flexible && (mixed || !amg)) fail(PRISM_INTERNAL, "flexible CG runs FP64 with AMG only");
    const int mode = flexible ? fcgMode(amg) : KM_BICGSTAB;
    const bool pre32 = mixed || mode == KM_FCG_PRE32;  // FP32 copy of the hierarchy
    w.ensure(A.nslices * 32, A.nnz_padded, mixed);
    const int n = A.n;
    const int gn = ceil_div(n, BS);
    // The iteration runs on A64 (FP64) / M32 (FP32) for the unknown X:
    // Jacobi: A' = A D^-1, X = D x (unscaled at the end); AMG: A itself, X = x.
    const bool scaled = amg == nullptr;
    SellMatrix A64 = A;
    double* X = x;
    const float* M32 = nullptr;
    if (scaled) {
        dinv_kernel<<<gn, BS, 0, s>>>(n, A.diag_pos, A.vals, w.dinv.p, x, w.xs.p); countLaunch();
        int sgrid = std::min<int64_t>((A.nnz_padded + BS - 1) / BS, NUM_SMS * 32);
        scale_kernel<double><<<sgrid, BS, 0, s>>>(A.nnz_padded, A.col, A.vals, w.dinv.p, w.As.p); countLaunch();
        if (mixed) {
            scale_kernel<float><<<sgrid, BS, 0, s>>>(A.nnz_padded, A.col, A.vals, w.dinv.p, w.As32.p); countLaunch();
        }
        PB_LAUNCH("bicgstab scaling");
        A64.vals = w.As.p;
        X = w.xs.p;
        M32 = w.As32.p;
    } else {
        if (!rowptr || !col) fail(PRISM_INTERNAL, "AMG preconditioner without a CSR pattern");
        w.ensurePrec(pre32);
        VerboseTimer vt("amg setup", s);
        amg->setup(A, rowptr, col, pre32, s);
        M32 = amg->vals32();
    }
    VerboseTimer vt_solve(mixed ? "bicgstab fp32+fp64" : flexible ? "fcg fp64" : "bicgstab fp64", s);
    auto finish = [&] {
        if (scaled) {
            unscale_kernel<<<gn, BS, 0, s>>>(n, w.dinv.p, w.xs.p, x); countLaunch();
            PB_LAUNCH("bicgstab unscale");
        }
    };
    KrylovOut out;
    if (!mixed) {
        Vecs<double> V{X, w.r.p, w.r0.p, w.p.p, w.v.p, w.s.p, w.t.p};
        // accurate-residual restarts: the recursive residual drifts from b - A x
        for (int pass = 0; pass < 4; ++pass) {
            KrylovOut o = runBicgstab<double>(A, A64.vals, b, V, false, tol, maxit, w, s, amg, w.y.p, w.z.p, mode);
            if (w.host_state->done == 4) PB_CUDA(cudaMemsetAsync(X, 0, n * sizeof(double), s));  // b = 0: x = 0
            out.iterations += o.iterations;
            out.status = o.status;
            maxit -= o.iterations;
            finish();
            spmv(A, x, w.tmp.p, s);
            double rb[2];
            refine_residual_kernel<<<vecGrid(n), BS, 0, s>>>(n, w.tmp.p, b, reinterpret_cast<float*>(w.s.p),
                                                             w.partials.p, w.counter.p, w.scal.p); countLaunch();
            PB_CUDA(cudaMemcpyAsync(rb, w.scal.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
            PB_CUDA(cudaStreamSynchronize(s));
            out.rel_residual = rb[1] > 0 ? std::sqrt(rb[0] / rb[1]) : 0.0;
            if (o.status != PRISM_OK || out.rel_residual <= 10 * tol || maxit <= 0 || rb[1] == 0) break;
        }
        if (verbose())
            std::fprintf(stderr, "[prism] %s fp64 n=%d: %lld iterations, rel residual %.3e, status %d\n",
                         flexible ? "fcg" : "bicgstab", n, out.iterations, out.rel_residual, out.status);
        return out;
    }
    // mixed precision: FP32 BiCGSTAB with FP64 reliable updates of X and r
    const double delta = (inner_tol > 0.0 && inner_tol < 1.0) ? inner_tol : 0.1;
    KState* S = w.state.p;
    KState init{};
    init.maxit = maxit;
    init.reliable = 1;
    init.delta2 = delta * delta;
    PB_CUDA(cudaMemcpyAsync(S, &init, sizeof(KState), cudaMemcpyHostToDevice, s));
    const int vg = vecGrid(n);
    auto reliable = [&](int first) {
        if (!first) {
            flush_kernel<<<gn, BS, 0, s>>>(n, X, w.x32.p); countLaunch();
        }
        spmv(A64, X, w.tmp.p, s);
        reliable_kernel<<<vg, BS, 0, s>>>(n, w.tmp.p, b, w.r64.p, w.r32.p, w.r032.p, w.p32.p, w.v32.p, first, tol,
                                          w.partials.p, w.counter.p, S); countLaunch();
        PB_LAUNCH("reliable update");
        PB_CUDA(cudaMemcpyAsync(w.host_state, S, sizeof(KState), cudaMemcpyDeviceToHost, s));
        PB_CUDA(cudaStreamSynchronize(s));
        if (verboseLevel() >= 2)
            std::fprintf(stderr, "[prism] mixed %s at iteration %lld: true rel residual %.3e, done %d\n",
                         first ? "restart" : "reliable update", w.host_state->iter,
                         w.host_state->bb > 0 ? std::sqrt(w.host_state->rr / w.host_state->bb) : 0.0,
                         w.host_state->done);
        return w.host_state->done;
    };
    fill_zero_f<<<gn, BS, 0, s>>>(n, w.x32.p); countLaunch();
    int done = reliable(1);
    int restarts = 0, n_reliable = 0, stalls = 0;
    long long batch = 8;
    // iterations of the current segment (since the last reliable update or restart) and the
    // longest segment so far: a segment far longer than every earlier one has stalled (the
    // FP32 recurrence stops reducing its residual), and restarting it from the current
    // FP64 solution recovers the convergence rate
    long long seg_start = 0, longest = 0;
    Vecs<float> V32{w.x32.p, w.r32.p, w.r032.p, w.p32.p, w.v32.p, w.s32.p, w.t32.p};
    bool first = true;
    while (done == 0) {
        iterate<float>(A, M32, V32, amg, w.y32.p, w.z32.p, batch, first, w, s);
        first = false;
        PB_LAUNCH("bicgstab fp32 iteration");
        PB_CUDA(cudaMemcpyAsync(w.host_state, S, sizeof(KState), cudaMemcpyDeviceToHost, s));
        PB_CUDA(cudaStreamSynchronize(s));
        done = w.host_state->done;
        const long long seg = w.host_state->iter - seg_start;
        if (done == 0) {
            if (seg > std::max(kStallMin, kStallFactor * longest) && stalls < 20) {
                ++stalls;
                longest = std::max(longest, seg);
                seg_start = w.host_state->iter;
                flush_kernel<<<gn, BS, 0, s>>>(n, X, w.x32.p); countLaunch();
                done = reliable(1);
                continue;
            }
            batch = std::min<long long>(batch * 2, 64);
            continue;
        }
        longest = std::max(longest, seg);
        seg_start = w.host_state->iter;
        if (done == 6) {
            ++n_reliable;
            if (restartOnUpdate()) {
                flush_kernel<<<gn, BS, 0, s>>>(n, X, w.x32.p); countLaunch();
                done = reliable(1);
            } else {
                done = reliable(0);
            }
            continue;
        }
        if (done == 3) {  // breakdown of the recurrence: flush and restart from the current x
            if (++restarts > 20) break;
            flush_kernel<<<gn, BS, 0, s>>>(n, X, w.x32.p); countLaunch();
            done = reliable(1);
            continue;
        }
        if (done == 5) {  // the FP32 recurrence overflowed: drop its correction, restart from X
            if (++restarts > 20) break;
            fill_zero_f<<<gn, BS, 0, s>>>(n, w.x32.p); countLaunch();
            done = reliable(1);
            continue;
        }
    }
    if (done == 2 || done == 3) {
        flush_kernel<<<gn, BS, 0, s>>>(n, X, w.x32.p); countLaunch();
    }
    out.iterations = w.host_state->iter;
    out.status = done == 1 || done == 4 ? PRISM_OK
                 : done == 2           ? PRISM_NOT_CONVERGED
                 : done == 5           ? PRISM_NONFINITE
                                       : PRISM_BREAKDOWN;
    out.rel_residual = w.host_state->bb > 0 ? std::sqrt(w.host_state->rr / w.host_state->bb) : 0.0;
    if (done == 4) PB_CUDA(cudaMemsetAsync(X, 0, n * sizeof(double), s));
    finish();
    if (verbose())
        std::fprintf(stderr, "[prism] bicgstab fp32+fp64 n=%d: %lld iterations, %d reliable updates, %d restarts, "
                     "%d stalled segments restarted, rel residual %.3e, status %d\n", n, out.iterations, n_reliable,
                     restarts, stalls, out.rel_residual, out.status);
    return out;
}

int profBegin(int kind, bool fp32, double bytes, cudaStream_t s) {
    if (!g_prof.on || (int)g_prof.samples.size() >= g_prof.max_samples) return -1;
    Sample smp{g_prof.get(), g_prof.get(), kind, fp32, bytes, false};
    PB_CUDA(cudaEventRecord(smp.a, s));
    g_prof.samples.push_back(smp);
    return (int)g_prof.samples.size() - 1;
}
void profEnd(int slot, cudaStream_t s) {
    if (slot < 0 || slot >= (int)g_prof.samples.size()) return;
    PB_CUDA(cudaEventRecord(g_prof.samples[slot].b, s));
    g_prof.samples[slot].closed = true;
}

void profileStart(int max_samples) {
    for (auto& smp : g_prof.samples) {
        g_prof.pool.push_back(smp.a);
        g_prof.pool.push_back(smp.b);
    }
    g_prof.samples.clear();
    g_prof.max_samples = max_samples > 0 ? max_samples : 4096;
    g_prof.launches0 = launchCounter().load();
    g_prof.graphs0 = graphLaunchCounter().load();
    g_prof.on = true;
}

void profileStop(PrismProfile* out) {
    std::memset(out, 0, sizeof(*out));
    g_prof.on = false;
    out->kernel_launches = launchCounter().load() - g_prof.launches0;
    out->graph_launches = graphLaunchCounter().load() - g_prof.graphs0;
    for (auto& smp : g_prof.samples) {
        if (!smp.closed) continue;
        PB_CUDA(cudaEventSynchronize(smp.b));
        float ms = 0.f;
        PB_CUDA(cudaEventElapsedTime(&ms, smp.a, smp.b));
        if (smp.kind == PROF_AMG_DOWN) {
            auto [l, t, b] = smp.fp32 ? std::tie(out->amg32_down_launches, out->amg32_down_ms, out->amg32_down_bytes)
                                       : std::tie(out->amg_down_launches, out->amg_down_ms, out->amg_down_bytes);
            l++;
            t += ms;
            b += smp.bytes;
        } else if (smp.kind == PROF_AMG_POST) {
            auto [l, t, b] = smp.fp32 ? std::tie(out->amg32_post_launches, out->amg32_post_ms, out->amg32_post_bytes)
                                       : std::tie(out->amg_post_launches, out->amg_post_ms, out->amg_post_bytes);
            l++;
            t += ms;
            b += smp.bytes;
        } else if (smp.kind == PROF_FCG_SPMV) {
            out->fcg_launches++;
            out->fcg_ms += ms;
            out->fcg_bytes += smp.bytes;
        } else if (smp.fp32) {
            out->fp32_launches++;
            out->fp32_ms += ms;
            out->fp32_bytes += smp.bytes;
        } else {
            out->fp64_launches++;
            out->fp64_ms += ms;
            out->fp64_bytes += smp.bytes;
        }
    }
}

void jacobiStep(const SellMatrix& A, const double* b, double* x, KrylovWork& w, cudaStream_t s) {
    w.ensure(A.nslices * 32, A.nnz_padded, false);
    jacobi_kernel<<<spmvGrid(A.nslices), BS, 0, s>>>(A.nslices, A.n, A.sl_off, A.col, A.vals, A.diag_pos, b, x,
                                                      w.tmp.p); countLaunch();
    PB_LAUNCH("jacobi_kernel");
    PB_CUDA(cudaMemcpyAsync(x, w.tmp.p, A.n * sizeof(double), cudaMemcpyDeviceToDevice, s));
}

void explicitUpdate(const SellMatrix& A, const double* b, const double* x, double* xnew, cudaStream_t s) {
    explicit_kernel<<<spmvGrid(A.nslices), BS, 0, s>>>(A.nslices, A.n, A.sl_off, A.col, A.vals, A.diag_pos, b, x,
                                                        xnew); countLaunch();
    PB_LAUNCH("explicit_kernel");
}

double scaledResidual(const SellMatrix& A, const double* b, const double* x, KrylovWork& w, cudaStream_t s) {
    w.ensure(A.nslices * 32, A.nnz_padded, false);
    resid_kernel<<<waveGrid(resid_kernel, ceil_div(A.nslices, WARPS)), BS, 0, s>>>(A.nslices, A.n, A.sl_off, A.col, A.vals, A.diag_pos, b, x,
                                                     w.partials.p, w.counter.p, w.scal.p); countLaunch();
    PB_LAUNCH("resid_kernel");
    double h[3];
    PB_CUDA(cudaMemcpyAsync(h, w.scal.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
    if (h[2] != 0.0) return NAN;
    return h[0] / (h[1] + EPSILON);
}

double offDiagonalRatio(const SellMatrix& A, KrylovWork& w, cudaStream_t s) {
    w.ensure(A.nslices * 32, A.nnz_padded, false);
    offdiag_ratio_kernel<<<waveGrid(offdiag_ratio_kernel, ceil_div(A.nslices, WARPS)), BS, 0, s>>>(
        A.nslices, A.n, A.sl_off, A.col, A.vals, w.partials.p, w.counter.p, w.scal.p); countLaunch();
    PB_LAUNCH("offdiag_ratio_kernel");
    double h = 0.0;
    PB_CUDA(cudaMemcpyAsync(&h, w.scal.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
    return h;
}

// ---------------------------------------------------------------- solves inside a CUDA graph
namespace {

enum { PH_INIT = 0, PH_ITER = 1, PH_CHECK = 2, PH_DONE = 3 };
constexpr int GRAPH_UNROLL = 4;  // BiCGSTAB iterations per pass of the device loop

__device__ __forceinline__ double nanValue() { return __longlong_as_double(0x7ff8000000000000LL); }

__global__ void ctl_solve_begin_kernel(SolveCtl* c, long long n_iter, double eps, long long kmax, double tol,
                                       cudaGraphConditionalHandle ho) {
    if (threadIdx.x) return;
    cudaGraphSetConditional(ho, 1u);
    SolveCtl z{};
    z.n_iter = n_iter;
    z.eps = eps;
    z.kmax = kmax;
    z.tol = tol;
    z.status = PRISM_OK;
    z.kstatus = PRISM_OK;
    z.phase = PH_DONE;
    *c = z;
}

__global__ void ctl_init_res_kernel(SolveCtl* c, const double* scal) {
    if (threadIdx.x) return;
    c->init_res = scal[2] != 0.0 ? nanValue() : scal[0] / (scal[1] + EPSILON);
}

// a fresh KState for one pass (runBicgstab's initial state: zeros, the iteration cap)
__device__ void resetState(KState* S, long long maxit) {
    KState z{};
    z.maxit = maxit;
    *S = z;
}

// start of one bicgstab() call: its first pass, and the device loop switched on
__global__ void ctl_krylov_begin_kernel(SolveCtl* c, KState* S, cudaGraphConditionalHandle hk) {
    if (threadIdx.x) return;
    c->maxit_left = c->kmax;
    c->pass = 0;
    c->restarts = 0;
    c->kstatus = PRISM_OK;
    c->krylov_rel = 0.0;
    c->guard = 0;
    c->phase = PH_INIT;
    resetState(S, c->kmax);
    cudaGraphSetConditional(hk, 1u);
}

// first node of a loop pass: which phase body runs
__global__ void ctl_phase_kernel(const SolveCtl* c, cudaGraphConditionalHandle hi, cudaGraphConditionalHandle ht,
                                 cudaGraphConditionalHandle hc) {
    if (threadIdx.x) return;
    cudaGraphSetConditional(hi, c->phase == PH_INIT ? 1u : 0u);
    cudaGraphSetConditional(ht, c->phase == PH_ITER ? 1u : 0u);
    cudaGraphSetConditional(hc, c->phase == PH_CHECK ? 1u : 0u);
}

// One transition of bicgstab()'s control flow (runBicgstab's batches, restarts
// and accurate-residual passes), after the body of the current phase has run.
__global__ void ctl_krylov_step_kernel(SolveCtl* c, KState* S, const double* scal, long long guard_max,
                                       cudaGraphConditionalHandle hk) {
    if (threadIdx.x) return;
    if (c->phase == PH_INIT) {
        c->phase = PH_ITER;
    } else if (c->phase == PH_ITER) {
        const int d = S->done;
        if (d == 3) {  // restart from the current x
            if (++c->restarts > 20) {
                c->kstatus = PRISM_BREAKDOWN;
                c->phase = PH_CHECK;
            } else {
                c->phase = PH_INIT;
            }
        } else if (d != 0) {
            c->kstatus = d == 2 ? PRISM_NOT_CONVERGED : d == 5 ? PRISM_NONFINITE : PRISM_OK;
            c->phase = PH_CHECK;
        }
    } else if (c->phase == PH_CHECK) {
        const double rb0 = scal[0], rb1 = scal[1];
        c->krylov_rel = rb1 > 0 ? sqrt(rb0 / rb1) : 0.0;
        c->krylov_iterations += S->iter;
        c->maxit_left -= S->iter;
        c->pass += 1;
        if (c->kstatus != PRISM_OK || c->krylov_rel <= 10 * c->tol || c->maxit_left <= 0 || rb1 == 0 || c->pass >= 4) {
            c->phase = PH_DONE;
        } else {
            resetState(S, c->maxit_left);
            c->restarts = 0;
            c->kstatus = PRISM_OK;
            c->phase = PH_INIT;
        }
    }
    if (++c->guard > guard_max && c->phase != PH_DONE) {  // safety net: the caps above end every solve first
        c->kstatus = PRISM_NOT_CONVERGED;
        c->phase = PH_DONE;
    }
    cudaGraphSetConditional(hk, c->phase != PH_DONE ? 1u : 0u);
}

// b = 0 ends a pass with x = 0 (bicgstab()'s memset on done == 4)
__global__ void zero_if_rhs_zero_kernel(int n, double* x, const KState* S) {
    if (S->done != 4) return;
    for (int i = blockIdx.x * BS + threadIdx.x; i < n; i += gridDim.x * BS) x[i] = 0.0;
}

__global__ void ctl_outer_step_kernel(SolveCtl* c, const double* scal, cudaGraphConditionalHandle ho) {
    if (threadIdx.x) return;
    const double cur = scal[2] != 0.0 ? nanValue() : scal[0] / (scal[1] + EPSILON);
    c->cur_res = cur;
    if (c->kstatus != PRISM_OK && c->status == PRISM_OK) c->status = c->kstatus;
    if (isnan(cur)) c->status = PRISM_NONFINITE;
    c->outer += 1;
    const bool conv = cur < c->eps;
    if (conv) c->converged = 1;
    cudaGraphSetConditional(ho, (!conv && c->outer < c->n_iter) ? 1u : 0u);
}

}  // namespace

cudaStream_t CaptureStreams::at(int depth) {
    if (depth < 0 || depth >= 3) fail(PRISM_INTERNAL, "conditional nodes nested too deep");
    if (!s[depth]) PB_CUDA(cudaStreamCreateWithFlags(&s[depth], cudaStreamNonBlocking));
    return s[depth];
}
CaptureStreams::~CaptureStreams() {
    for (auto& x : s)
        if (x) cudaStreamDestroy(x);
}

bool capturing(cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &st) != cudaSuccess) return false;
    return st == cudaStreamCaptureStatusActive;
}

cudaGraphConditionalHandle createConditional(cudaStream_t s, unsigned dflt) {
    cudaStreamCaptureStatus st;
    unsigned long long id;
    cudaGraph_t g;
    const cudaGraphNode_t* deps;
    size_t nd;
    PB_CUDA(cudaStreamGetCaptureInfo(s, &st, &id, &g, &deps, &nd));
    if (st != cudaStreamCaptureStatusActive) fail(PRISM_INTERNAL, "conditional handle outside a capture");
    cudaGraphConditionalHandle h;
    PB_CUDA(cudaGraphConditionalHandleCreate(&h, g, dflt, cudaGraphCondAssignDefault));
    return h;
}

void beginConditional(cudaStream_t s, cudaGraphConditionalNodeType type, cudaGraphConditionalHandle h,
                      cudaStream_t body) {
    cudaStreamCaptureStatus st;
    unsigned long long id;
    cudaGraph_t g;
    const cudaGraphNode_t* deps;
    size_t nd;
    PB_CUDA(cudaStreamGetCaptureInfo(s, &st, &id, &g, &deps, &nd));
    if (st != cudaStreamCaptureStatusActive) fail(PRISM_INTERNAL, "conditional node outside a capture");
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = type;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    PB_CUDA(cudaGraphAddNode(&node, g, deps, nd, &p));
    PB_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    PB_CUDA(cudaStreamBeginCaptureToGraph(body, p.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeRelaxed));
}

void endConditional(cudaStream_t body) {
    cudaGraph_t g;
    PB_CUDA(cudaStreamEndCapture(body, &g));
}

void emitSolveBegin(SolveCtl* ctl, long long n_iter, double eps, long long kmax, double tol,
                    cudaGraphConditionalHandle outer, cudaStream_t s) {
    ctl_solve_begin_kernel<<<1, 32, 0, s>>>(ctl, n_iter, eps, kmax, tol, outer); countLaunch();
}

void emitResidual(const SellMatrix& A, const double* b, const double* x, KrylovWork& w, cudaStream_t s) {
    resid_kernel<<<waveGrid(resid_kernel, ceil_div(A.nslices, WARPS)), BS, 0, s>>>(
        A.nslices, A.n, A.sl_off, A.col, A.vals, A.diag_pos, b, x, w.partials.p, w.counter.p, w.scal.p); countLaunch();
}

void emitInitResidual(SolveCtl* ctl, KrylovWork& w, cudaStream_t s) {
    ctl_init_res_kernel<<<1, 32, 0, s>>>(ctl, w.scal.p); countLaunch();
}

void emitOuterStep(SolveCtl* ctl, KrylovWork& w, cudaGraphConditionalHandle outer, cudaStream_t s) {
    ctl_outer_step_kernel<<<1, 32, 0, s>>>(ctl, w.scal.p, outer); countLaunch();
}

// bicgstab() (FP64) with its host loops turned into a device loop:
//   WHILE (phase != DONE) { IF INIT {r = b - A x; init} IF ITER {GRAPH_UNROLL iterations}
//                           IF CHECK {x = 0 if b = 0; unscale; accurate residual} controller }
// The kernels and their order are those of the eager path, so the results are the same.
void emitBicgstab(const SellMatrix& A, const double* b, double* x, double tol, long long maxit, KrylovWork& w,
                  cudaStream_t s, Amg* amg, const int* rowptr, const int* col, SolveCtl* ctl, CaptureStreams& cs,
                  int depth, bool flexible) {
    if (flexible && !amg) fail(PRISM_INTERNAL, "flexible CG runs with AMG only");
    const int mode = flexible ? fcgMode(amg) : KM_BICGSTAB;
    w.ensure(A.nslices * 32, A.nnz_padded, false);
    const int n = A.n, gn = ceil_div(n, BS);
    const bool scaled = amg == nullptr;
    SellMatrix A64 = A;
    double* X = x;
    if (scaled) {
        dinv_kernel<<<gn, BS, 0, s>>>(n, A.diag_pos, A.vals, w.dinv.p, x, w.xs.p); countLaunch();
        int sgrid = std::min<int64_t>((A.nnz_padded + BS - 1) / BS, NUM_SMS * 32);
        scale_kernel<double><<<sgrid, BS, 0, s>>>(A.nnz_padded, A.col, A.vals, w.dinv.p, w.As.p); countLaunch();
        A64.vals = w.As.p;
        X = w.xs.p;
    } else {
        if (!rowptr || !col) fail(PRISM_INTERNAL, "AMG preconditioner without a CSR pattern");
        w.ensurePrec(mode == KM_FCG_PRE32);
        amg->setup(A, rowptr, col, mode == KM_FCG_PRE32, s);
    }
    KState* S = w.state.p;
    Vecs<double> V{X, w.r.p, w.r0.p, w.p.p, w.v.p, w.s.p, w.t.p};
    const int vg = vecGrid(n), sg = sliceGrid(A.nslices);
    const long long guard_max = 4 * (maxit / GRAPH_UNROLL + 64) + 256;
    cudaStream_t body = cs.at(depth), sub = cs.at(depth + 1);
    cudaGraphConditionalHandle hk = createConditional(s, 0);
    ctl_krylov_begin_kernel<<<1, 32, 0, s>>>(ctl, S, hk); countLaunch();
    beginConditional(s, cudaGraphCondTypeWhile, hk, body);
    cudaGraphConditionalHandle hi = createConditional(body, 0), ht = createConditional(body, 0),
                               hc = createConditional(body, 0);
    ctl_phase_kernel<<<1, 32, 0, body>>>(ctl, hi, ht, hc); countLaunch();
    beginConditional(body, cudaGraphCondTypeIf, hi, sub);
    spmv_kernel<double, 0><<<sg, BS, 0, sub>>>(A.nslices, n, A.sl_off, A.col, A64.vals, V.x, V.r, nullptr, nullptr,
                                               nullptr, nullptr); countLaunch();
    if (flexible) {
        fcg_init_kernel<<<vg, BS, 0, sub>>>(n, V.r, b, V.p, V.v, mode == KM_FCG_PRE32 ? w.y32.p : nullptr, tol,
                                            w.partials.p, w.counter.p, S); countLaunch();
    } else {
        init_kernel<double><<<vg, BS, 0, sub>>>(n, V.r, b, V.r0, V.p, V.v, 0, tol, w.partials.p, w.counter.p, S); countLaunch();
    }
    endConditional(sub);
    beginConditional(body, cudaGraphCondTypeIf, ht, sub);
    iterateAny<double>(A, A64.vals, V, amg, w.y.p, w.z.p, GRAPH_UNROLL, false, mode, w, sub);
    endConditional(sub);
    beginConditional(body, cudaGraphCondTypeIf, hc, sub);
    zero_if_rhs_zero_kernel<<<vg, BS, 0, sub>>>(n, X, S); countLaunch();
    if (scaled) {
        unscale_kernel<<<gn, BS, 0, sub>>>(n, w.dinv.p, w.xs.p, x); countLaunch();
    }
    spmv(A, x, w.tmp.p, sub);
    refine_residual_kernel<<<vg, BS, 0, sub>>>(n, w.tmp.p, b, reinterpret_cast<float*>(w.s.p), w.partials.p,
                                               w.counter.p, w.scal.p); countLaunch();
    endConditional(sub);
    ctl_krylov_step_kernel<<<1, 32, 0, body>>>(ctl, S, w.scal.p, guard_max, hk); countLaunch();
    endConditional(body);
}

}  // namespace pb
