// batched.cu -- many independent BiCGSTAB solves in one persistent launch.
//
// The systems are laid side by side as one block-diagonal SELL-32 matrix (a
// slice never straddles two systems). One cooperative kernel runs the whole
// solve: every phase sweeps the rows of the systems still iterating, with
// grid-wide barriers between phases, and every reduction is per system
// (warp/slice partial sums, then one block per system summing its partials in
// a fixed order: deterministic, no atomics on floating point). Per system:
//   * BiCGSTAB (the recurrences of bicgstab.cpp's Eigen solver) on A D^-1,
//     in FP32 with FP64 dot products when mixed, else in FP64;
//   * each inner solve stops when its residual has dropped by itol (or on a
//     breakdown, or after max_inner iterations); then an FP64 refinement step
//     x += D^-1 d, r = b - A x (FP64 matrix) decides: converged
//     (||r|| <= tol ||b||), failed (max_pass / maxit reached) or a new inner
//     solve on r.
// Systems finish independently: every block lists the systems in the state a
// phase works on (in shared memory, from the states), and each warp walks a
// contiguous run of their slices, so finished systems cost nothing.
// Launch shape (block size, lanes per row of the SpMV sweeps) is autotuned on
// the batch itself and kept with the plan.
#include <cooperative_groups.h>

#include <chrono>
#include <cmath>
#include <cstring>

#include "batched.h"

namespace cg = cooperative_groups;

namespace pb {

namespace {

constexpr int MAX_BLOCK = 512;

enum { S_INNER = 0, S_REFINE = 1, S_DONE = 2, S_FAILED = 3 };

struct BState {
    double rho, alpha, omega, beta, bb, tol2, rr64, rr0;
    long long iter;
    int state, fresh, pass, inner, status, stop;
};

template <typename T>
struct BP {
    int nprob, nslices;
    const int* slice_prob;
    const int* prob_slice0;
    const int* prob_n;
    const int* sl_off;
    const int* col;
    const double* A64;
    const T* A;  // column-scaled inner matrix A D^-1
    const double* b64;
    const double* dinv;
    double* x64;
    T *r, *r0, *p, *v, *s, *t, *d;
    double* cdot;  // 3 per chunk of the SpMV sweeps (nslices * lpr chunks)
    double* sdot;  // 2 per slice (update sweep)
    BState* st;
    int* ctl;  // [2 * buffer]: systems still active, systems waiting for refinement
    double tol2, itol2;
    int max_inner, max_pass, max_steps;
    long long maxit;
};

// Data written inside the launch by other blocks is read through L2 (ld.cg).
__device__ __forceinline__ int stateOf(const BState* st, int p) { return __ldcg(&st[p].state); }
__device__ __forceinline__ double ld(const double* a, int i) { return __ldcg(a + i); }
__device__ __forceinline__ float ld(const float* a, int i) { return __ldcg(a + i); }

__device__ __forceinline__ double warpSum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
// block-wide sums of a and b (valid in thread 0); sh holds 2 * MAX_BLOCK / 32 doubles
__device__ __forceinline__ void blockSum2(double& a, double& b, double* sh) {
    a = warpSum(a);
    b = warpSum(b);
    const int w = threadIdx.x >> 5;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
        sh[w] = a;
        sh[MAX_BLOCK / 32 + w] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ta = 0.0, tb = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            ta += sh[i];
            tb += sh[MAX_BLOCK / 32 + i];
        }
        a = ta;
        b = tb;
    }
}

// Sum over this row's SELL slots of val * xf(col), LPR adjacent lanes per row;
// the total is returned in every lane of the group.
template <int LPR, typename V, typename F>
__device__ __forceinline__ double rowDot(const int* sl_off, const int* col, const V* val, int row, int sub, F xf) {
    const int s = row >> 5;
    const int s0 = sl_off[s];
    const int width = (sl_off[s + 1] - s0) >> 5;
    const int bo = s0 + (row & 31);
    double sum = 0.0;
    for (int j = sub; j < width; j += LPR) {
        const int q = bo + 32 * j;
        sum += (double)val[q] * xf(col[q]);
    }
    if constexpr (LPR > 1) {
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    }
    return sum;
}

// Systems in state `want`, listed in every block's shared memory: ids[k] and
// the prefix pre[k] of their slice counts (pre[m] = total). Each block builds
// the same list from the states, so no extra grid barrier is needed.
template <typename T>
__device__ int buildList(const BP<T>& P, int want, int* pre, int* ids, int* tmp, int& m_out) {
    const int nt = blockDim.x, t = threadIdx.x;
    const int per = (P.nprob + nt - 1) / nt;
    const int k0 = min(t * per, P.nprob), k1 = min(k0 + per, P.nprob);
    int cnt = 0, sl = 0;
    for (int k = k0; k < k1; ++k)
        if (stateOf(P.st, k) == want) {
            ++cnt;
            sl += P.prob_slice0[k + 1] - P.prob_slice0[k];
        }
    __syncthreads();
    tmp[t] = cnt;
    tmp[nt + t] = sl;
    __syncthreads();
    if (t == 0) {
        int c = 0, q = 0;
        for (int i = 0; i < nt; ++i) {
            const int a = tmp[i], b = tmp[nt + i];
            tmp[i] = c;
            tmp[nt + i] = q;
            c += a;
            q += b;
        }
        tmp[2 * nt] = c;
        tmp[2 * nt + 1] = q;
    }
    __syncthreads();
    int c = tmp[t], q = tmp[nt + t];
    for (int k = k0; k < k1; ++k)
        if (stateOf(P.st, k) == want) {
            ids[c] = k;
            pre[c] = q;
            ++c;
            q += P.prob_slice0[k + 1] - P.prob_slice0[k];
        }
    const int m = tmp[2 * nt], total = tmp[2 * nt + 1];
    if (t == 0) pre[m] = total;
    __syncthreads();
    m_out = m;
    return total;
}
// list entry holding virtual slice v (pre[k] <= v < pre[k+1])
__device__ __forceinline__ int findEntry(const int* pre, int m, int v) {
    int lo = 0, hi = m;  // pre[lo] <= v < pre[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (pre[mid] <= v) lo = mid;
        else hi = mid;
    }
    return lo;
}

// A warp's contiguous run of list units (slices, or chunks of LPR per slice):
// tracks the system of the current unit so that per-system data is loaded once
// per run segment instead of once per unit.
struct Run {
    int v, vend;  // units [v, vend)
    int k, kend;  // list entry and the unit where it ends
    int pr, slice0, rows_end;
};
template <typename T>
__device__ __forceinline__ void runEnter(const BP<T>& P, const int* pre, const int* ids, int upu, Run& R) {
    R.pr = ids[R.k];
    R.kend = pre[R.k + 1] * upu;
    R.slice0 = P.prob_slice0[R.pr] - pre[R.k];
    R.rows_end = 32 * P.prob_slice0[R.pr] + P.prob_n[R.pr];
}
// upu: units per slice; returns false when the warp has no units
template <typename T>
__device__ __forceinline__ bool runStart(const BP<T>& P, const int* pre, const int* ids, int m, int total_units,
                                         int upu, int gwarp, int nwarps, Run& R) {
    const int per = (total_units + nwarps - 1) / nwarps;
    R.v = gwarp * per;
    R.vend = min(R.v + per, total_units);
    if (R.v >= R.vend) return false;
    R.k = findEntry(pre, m, R.v / upu);
    runEnter(P, pre, ids, upu, R);
    return true;
}
// advance to the system of unit R.v; true when the system changed
template <typename T>
__device__ __forceinline__ bool runSeek(const BP<T>& P, const int* pre, const int* ids, int upu, Run& R) {
    if (R.v < R.kend) return false;
    while (R.v >= pre[R.k + 1] * upu) ++R.k;
    runEnter(P, pre, ids, upu, R);
    return true;
}

// Row sums of US consecutive units (chunks of one system) starting at R.v:
// the slots of all units are walked together so that their loads overlap.
template <typename T, int LPR, int US, typename V, typename F>
__device__ __forceinline__ void spmvUnits(const BP<T>& P, const V* val, const Run& R, int nh, int lane, int* row,
                                          int* chunk, double* sum, F xf) {
    constexpr int RPC = 32 / LPR;
    const int sub = lane % LPR;
    int bo[US], w[US];
    int wmax = 0;
#pragma unroll
    for (int u = 0; u < US; ++u) {
        const int vu = R.v + (u < nh ? u : 0);
        const int slice = R.slice0 + vu / LPR;
        chunk[u] = slice * LPR + vu % LPR;
        row[u] = 32 * slice + (vu % LPR) * RPC + lane / LPR;
        const int s0 = P.sl_off[slice];
        w[u] = u < nh ? (P.sl_off[slice + 1] - s0) >> 5 : 0;
        bo[u] = s0 + (row[u] & 31);
        sum[u] = 0.0;
        wmax = max(wmax, w[u]);
    }
    for (int j = sub; j < wmax; j += LPR) {
#pragma unroll
        for (int u = 0; u < US; ++u)
            if (j < w[u]) {
                const int q = bo[u] + 32 * j;
                sum[u] += (double)val[q] * xf(P.col[q]);
            }
    }
    if constexpr (LPR > 1) {
#pragma unroll
        for (int u = 0; u < US; ++u)
#pragma unroll
            for (int o = LPR / 2; o > 0; o >>= 1) sum[u] += __shfl_xor_sync(0xffffffffu, sum[u], o);
    }
}

// At most 64 registers per thread (2 blocks of 512 per SM): the sweeps are
// latency-bound, so loads in flight (UR / US units per warp step) and
// occupancy matter more than registers.
template <typename T, int LPR>
__global__ void __launch_bounds__(MAX_BLOCK, 2) batch_kernel(const BP<T> P) {
    __shared__ double sh[2 * MAX_BLOCK / 32];
    extern __shared__ int lists[];  // pre (nprob + 1) | ids (nprob) | scan scratch (2 * blockDim + 2)
    int* pre = lists;
    int* ids = lists + P.nprob + 1;
    int* tmp = lists + 2 * P.nprob + 1;
    cg::grid_group grid = cg::this_grid();
    const int lane = threadIdx.x & 31;
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    constexpr int RPC = 32 / LPR;  // rows per chunk (one warp)
    constexpr int UR = 2;          // slices per warp step in the row sweeps
    constexpr int US = LPR == 1 ? 2 : 1;  // units per warp step in the SpMV sweeps
    Run R;

    for (int step = 0; step < P.max_steps; ++step) {
        const int cur = step & 1, nxt = cur ^ 1;
        const int n_active = __ldcg(&P.ctl[2 * cur]);
        const int n_refine = __ldcg(&P.ctl[2 * cur + 1]);
        if (n_active == 0) break;  // the same value in every thread: read after a grid barrier
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            P.ctl[2 * nxt] = 0;
            P.ctl[2 * nxt + 1] = 0;
        }
        int m;
        if (n_refine > 0) {
            const int total = buildList(P, S_REFINE, pre, ids, tmp, m);
            // R1: x += D^-1 d, d = 0 (systems waiting for refinement)
            if (runStart(P, pre, ids, m, total, 1, gwarp, nwarps, R)) {
                for (; R.v < R.vend; ++R.v) {
                    runSeek(P, pre, ids, 1, R);
                    const int r = 32 * (R.slice0 + R.v) + lane;
                    if (r >= R.rows_end) continue;
                    P.x64[r] = ld(P.x64, r) + P.dinv[r] * (double)ld(P.d, r);
                    P.d[r] = (T)0;
                }
            }
            grid.sync();
            // R2: r = b - A x in FP64; the inner residual starts from (T) r
            if (runStart(P, pre, ids, m, total * LPR, LPR, gwarp, nwarps, R)) {
                for (; R.v < R.vend; ++R.v) {
                    runSeek(P, pre, ids, LPR, R);
                    const int slice = R.slice0 + R.v / LPR;
                    const int chunk = slice * LPR + R.v % LPR;
                    const int row = 32 * slice + (R.v % LPR) * RPC + lane / LPR, sub = lane % LPR;
                    const bool valid = row < R.rows_end;
                    // every lane runs the same shuffles; padding rows hold zero values
                    const double ax = rowDot<LPR>(P.sl_off, P.col, P.A64, row, sub,
                                                  [&](int c) { return ld(P.x64, c); });
                    double t0 = 0.0, t1 = 0.0;
                    if (valid && sub == 0) {
                        const double r64 = P.b64[row] - ax;
                        const T rt = (T)r64;
                        P.r[row] = rt;
                        t0 = r64 * r64;
                        t1 = (double)rt * (double)rt;
                    }
                    t0 = warpSum(t0);
                    t1 = warpSum(t1);
                    if (lane == 0) {
                        P.cdot[3 * chunk] = t0;
                        P.cdot[3 * chunk + 1] = t1;
                    }
                }
            }
            grid.sync();
            // RED(R): converged, failed, or a new inner solve
            for (int pr = blockIdx.x; pr < P.nprob; pr += gridDim.x) {
                if (stateOf(P.st, pr) != S_REFINE) continue;
                const int c0 = P.prob_slice0[pr] * LPR, c1 = P.prob_slice0[pr + 1] * LPR;
                double a = 0.0, b = 0.0;
                for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
                    a += ld(P.cdot, 3 * c);
                    b += ld(P.cdot, 3 * c + 1);
                }
                blockSum2(a, b, sh);
                if (threadIdx.x == 0) {
                    BState& S = P.st[pr];
                    S.rr64 = a;
                    if (!isfinite(a)) {
                        S.status = PRISM_NONFINITE;
                        S.state = S_FAILED;
                    } else if (a <= P.tol2 * S.bb) {
                        S.state = S_DONE;
                    } else if (S.stop || S.pass >= P.max_pass || S.iter >= P.maxit) {
                        S.status = PRISM_NOT_CONVERGED;
                        S.state = S_FAILED;
                    } else {
                        S.pass += 1;
                        S.inner = 0;
                        S.rho = b;
                        S.rr0 = b;
                        S.alpha = 1.0;
                        S.omega = 1.0;
                        S.beta = 0.0;
                        S.tol2 = P.itol2 * b;
                        S.fresh = 1;
                        S.state = S_INNER;
                    }
                }
                __syncthreads();
            }
            grid.sync();
        }
        const int total = buildList(P, S_INNER, pre, ids, tmp, m);
        if (n_refine > 0) {
            // R3: fresh inner solves: r0 = r, p = v = 0
            if (runStart(P, pre, ids, m, total, 1, gwarp, nwarps, R)) {
                bool fresh = __ldcg(&P.st[R.pr].fresh);
                for (; R.v < R.vend; ++R.v) {
                    if (runSeek(P, pre, ids, 1, R)) fresh = __ldcg(&P.st[R.pr].fresh);
                    const int r = 32 * (R.slice0 + R.v) + lane;
                    if (!fresh || r >= R.rows_end) continue;
                    P.r0[r] = ld(P.r, r);
                    P.p[r] = (T)0;
                    P.v[r] = (T)0;
                }
            }
            grid.sync();
        }

        // ---- one BiCGSTAB iteration of every system in an inner solve
        // A: p = r + beta (p - omega v)          (UR slices per warp step: loads first, then stores)
        if (runStart(P, pre, ids, m, total, 1, gwarp, nwarps, R)) {
            double beta = __ldcg(&P.st[R.pr].beta), omega = __ldcg(&P.st[R.pr].omega);
            while (R.v < R.vend) {
                if (runSeek(P, pre, ids, 1, R)) {
                    beta = __ldcg(&P.st[R.pr].beta);
                    omega = __ldcg(&P.st[R.pr].omega);
                }
                const int nh = min(UR, min(R.kend, R.vend) - R.v);
                int rr[UR];
                T a0[UR], a1[UR], a2[UR];
#pragma unroll
                for (int u = 0; u < UR; ++u) {
                    rr[u] = 32 * (R.slice0 + R.v + u) + lane;
                    if (u < nh && rr[u] < R.rows_end) {
                        a0[u] = ld(P.r, rr[u]);
                        a1[u] = ld(P.p, rr[u]);
                        a2[u] = ld(P.v, rr[u]);
                    }
                }
#pragma unroll
                for (int u = 0; u < UR; ++u)
                    if (u < nh && rr[u] < R.rows_end)
                        P.p[rr[u]] = (T)((double)a0[u] + beta * ((double)a1[u] - omega * (double)a2[u]));
                R.v += nh;
            }
        }
        grid.sync();
        // B: v = A' p ; r0.v
        if (runStart(P, pre, ids, m, total * LPR, LPR, gwarp, nwarps, R)) {
            while (R.v < R.vend) {
                runSeek(P, pre, ids, LPR, R);
                const int nh = min(US, min(R.kend, R.vend) - R.v);
                int row[US], chunk[US];
                double sum[US];
                const int sub = lane % LPR;
                spmvUnits<T, LPR, US>(P, P.A, R, nh, lane, row, chunk, sum, [&](int c) { return (double)ld(P.p, c); });
#pragma unroll
                for (int u = 0; u < US; ++u) {
                    double t0 = 0.0;
                    if (u < nh && row[u] < R.rows_end && sub == 0) {
                        const T vt = (T)sum[u];
                        P.v[row[u]] = vt;
                        t0 = (double)ld(P.r0, row[u]) * (double)vt;
                    }
                    t0 = warpSum(t0);
                    if (lane == 0 && u < nh) P.cdot[3 * chunk[u]] = t0;
                }
                R.v += nh;
            }
        }
        grid.sync();
        // RED(B): alpha = rho / (r0.v)
        for (int pr = blockIdx.x; pr < P.nprob; pr += gridDim.x) {
            if (stateOf(P.st, pr) != S_INNER) continue;
            const int c0 = P.prob_slice0[pr] * LPR, c1 = P.prob_slice0[pr + 1] * LPR;
            double a = 0.0, b = 0.0;
            for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) a += ld(P.cdot, 3 * c);
            blockSum2(a, b, sh);
            if (threadIdx.x == 0) {
                BState& S = P.st[pr];
                const double alpha = S.rho / a;
                if (a == 0.0 || !isfinite(alpha)) {
                    S.state = S_REFINE;  // breakdown: refine and restart
                } else {
                    S.alpha = alpha;
                }
            }
            __syncthreads();
        }
        grid.sync();
        // D: s = r - alpha v   (systems that broke down in RED(B) are skipped from here on)
        if (runStart(P, pre, ids, m, total, 1, gwarp, nwarps, R)) {
            bool on = stateOf(P.st, R.pr) == S_INNER;
            double alpha = __ldcg(&P.st[R.pr].alpha);
            while (R.v < R.vend) {
                if (runSeek(P, pre, ids, 1, R)) {
                    on = stateOf(P.st, R.pr) == S_INNER;
                    alpha = __ldcg(&P.st[R.pr].alpha);
                }
                const int nh = min(UR, min(R.kend, R.vend) - R.v);
                if (on) {
                    int rr[UR];
                    T a0[UR], a1[UR];
#pragma unroll
                    for (int u = 0; u < UR; ++u) {
                        rr[u] = 32 * (R.slice0 + R.v + u) + lane;
                        if (u < nh && rr[u] < R.rows_end) {
                            a0[u] = ld(P.r, rr[u]);
                            a1[u] = ld(P.v, rr[u]);
                        }
                    }
#pragma unroll
                    for (int u = 0; u < UR; ++u)
                        if (u < nh && rr[u] < R.rows_end) P.s[rr[u]] = (T)((double)a0[u] - alpha * (double)a1[u]);
                }
                R.v += nh;
            }
        }
        grid.sync();
        // E: t = A' s ; t.s, t.t
        if (runStart(P, pre, ids, m, total * LPR, LPR, gwarp, nwarps, R)) {
            bool on = stateOf(P.st, R.pr) == S_INNER;
            while (R.v < R.vend) {
                if (runSeek(P, pre, ids, LPR, R)) on = stateOf(P.st, R.pr) == S_INNER;
                const int nh = min(US, min(R.kend, R.vend) - R.v);
                if (on) {  // the same system in the whole warp
                    int row[US], chunk[US];
                    double sum[US];
                    const int sub = lane % LPR;
                    spmvUnits<T, LPR, US>(P, P.A, R, nh, lane, row, chunk, sum,
                                          [&](int c) { return (double)ld(P.s, c); });
#pragma unroll
                    for (int u = 0; u < US; ++u) {
                        double t0 = 0.0, t1 = 0.0;
                        if (u < nh && row[u] < R.rows_end && sub == 0) {
                            const T tt = (T)sum[u];
                            P.t[row[u]] = tt;
                            t0 = (double)tt * (double)ld(P.s, row[u]);
                            t1 = (double)tt * (double)tt;
                        }
                        t0 = warpSum(t0);
                        t1 = warpSum(t1);
                        if (lane == 0 && u < nh) {
                            P.cdot[3 * chunk[u]] = t0;
                            P.cdot[3 * chunk[u] + 1] = t1;
                        }
                    }
                }
                R.v += nh;
            }
        }
        grid.sync();
        // RED(E): omega = (t.s) / (t.t)
        for (int pr = blockIdx.x; pr < P.nprob; pr += gridDim.x) {
            if (stateOf(P.st, pr) != S_INNER) continue;
            const int c0 = P.prob_slice0[pr] * LPR, c1 = P.prob_slice0[pr + 1] * LPR;
            double a = 0.0, b = 0.0;
            for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
                a += ld(P.cdot, 3 * c);
                b += ld(P.cdot, 3 * c + 1);
            }
            blockSum2(a, b, sh);
            if (threadIdx.x == 0) P.st[pr].omega = b > 0.0 ? a / b : 0.0;
            __syncthreads();
        }
        grid.sync();
        // G: d += alpha p + omega s ; r = s - omega t ; r0.r, r.r per slice
        if (runStart(P, pre, ids, m, total, 1, gwarp, nwarps, R)) {
            bool on = stateOf(P.st, R.pr) == S_INNER;
            double alpha = __ldcg(&P.st[R.pr].alpha), omega = __ldcg(&P.st[R.pr].omega);
            while (R.v < R.vend) {
                if (runSeek(P, pre, ids, 1, R)) {
                    on = stateOf(P.st, R.pr) == S_INNER;
                    alpha = __ldcg(&P.st[R.pr].alpha);
                    omega = __ldcg(&P.st[R.pr].omega);
                }
                const int nh = min(UR, min(R.kend, R.vend) - R.v);
                if (on) {  // the same system in the whole warp
                    int rr[UR];
                    T a0[UR], a1[UR], a2[UR], a3[UR], a4[UR];
                    bool ok[UR];
#pragma unroll
                    for (int u = 0; u < UR; ++u) {
                        rr[u] = 32 * (R.slice0 + R.v + u) + lane;
                        ok[u] = u < nh && rr[u] < R.rows_end;
                        if (ok[u]) {
                            a0[u] = ld(P.s, rr[u]);
                            a1[u] = ld(P.d, rr[u]);
                            a2[u] = ld(P.p, rr[u]);
                            a3[u] = ld(P.t, rr[u]);
                            a4[u] = ld(P.r0, rr[u]);
                        }
                    }
#pragma unroll
                    for (int u = 0; u < UR; ++u) {
                        double t0 = 0.0, t1 = 0.0;
                        if (ok[u]) {
                            const double si = (double)a0[u];
                            P.d[rr[u]] = (T)((double)a1[u] + alpha * (double)a2[u] + omega * si);
                            const T rt = (T)(si - omega * (double)a3[u]);
                            P.r[rr[u]] = rt;
                            t0 = (double)a4[u] * (double)rt;
                            t1 = (double)rt * (double)rt;
                        }
                        t0 = warpSum(t0);
                        t1 = warpSum(t1);
                        if (lane == 0 && u < nh) {
                            P.sdot[2 * (R.slice0 + R.v + u)] = t0;
                            P.sdot[2 * (R.slice0 + R.v + u) + 1] = t1;
                        }
                    }
                }
                R.v += nh;
            }
        }
        grid.sync();
        // RED(G): next beta, inner convergence; every system is counted for the next step
        for (int pr = blockIdx.x; pr < P.nprob; pr += gridDim.x) {
            const int stt = stateOf(P.st, pr);
            if (stt == S_INNER) {
                const int c0 = P.prob_slice0[pr], c1 = P.prob_slice0[pr + 1];
                double a = 0.0, b = 0.0;
                for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
                    a += ld(P.sdot, 2 * c);
                    b += ld(P.sdot, 2 * c + 1);
                }
                blockSum2(a, b, sh);
                if (threadIdx.x == 0) {
                    BState& S = P.st[pr];
                    S.fresh = 0;
                    S.iter += 1;
                    S.inner += 1;
                    if (!isfinite(a) || !isfinite(b)) {
                        S.state = S_REFINE;
                    } else if (b <= S.tol2 || S.inner >= P.max_inner || S.omega == 0.0 ||
                               fabs(a) < EPSILON * EPSILON * S.rr0) {
                        S.state = S_REFINE;
                    } else if (S.iter >= P.maxit) {
                        S.stop = 1;
                        S.state = S_REFINE;
                    } else {
                        S.beta = (a / S.rho) * (S.alpha / S.omega);
                        S.rho = a;
                    }
                }
                __syncthreads();
            }
            if (threadIdx.x == 0) {
                const int now = P.st[pr].state;
                if (now == S_INNER || now == S_REFINE) atomicAdd(&P.ctl[2 * nxt], 1);
                if (now == S_REFINE) atomicAdd(&P.ctl[2 * nxt + 1], 1);
            }
        }
        grid.sync();
    }
}

// ---------------------------------------------------------------- setup kernels
constexpr int BS = 256;
inline int grid(int64_t n) { return std::max(1, ceil_div(n, BS)); }

__global__ void shift_kernel(int64_t n, const int* in, int add, int* out) {
    for (int64_t i = blockIdx.x * (int64_t)BS + threadIdx.x; i < n; i += (int64_t)gridDim.x * BS) out[i] = in[i] + add;
}
__global__ void fill_int_kernel(int n, int value, int* out) {
    int i = blockIdx.x * BS + threadIdx.x;
    if (i < n) out[i] = value;
}
// D^-1 of every row (1 on padding rows)
// one system's buffers and its place in the concatenated ones
struct CopyEntry {
    const double* vals;
    const double* b;
    double* x;
    long long nnz, nnz_off, row_off;
    int n;
};
// gather (dir 0: systems -> concatenated values, b, x) or scatter (dir 1: x back);
// blockIdx.y is the system, blockIdx.x strides within it
__global__ void batch_copy_kernel(const CopyEntry* tab, int dir, double* A64, double* b64, double* x64) {
    const CopyEntry e = tab[blockIdx.y];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x, stride = (long long)gridDim.x * blockDim.x;
    if (dir == 0) {
        for (long long i = t; i < e.nnz; i += stride) A64[e.nnz_off + i] = e.vals[i];
        for (long long i = t; i < e.n; i += stride) {
            b64[e.row_off + i] = e.b[i];
            x64[e.row_off + i] = e.x[i];
        }
    } else {
        for (long long i = t; i < e.n; i += stride) e.x[i] = x64[e.row_off + i];
    }
}

__global__ void batch_dinv_kernel(int nrows, const int* diag, const double* A64, double* dinv) {
    int r = blockIdx.x * BS + threadIdx.x;
    if (r >= nrows) return;
    const int q = diag[r];
    const double dd = q >= 0 ? A64[q] : 0.0;
    dinv[r] = dd != 0.0 ? 1.0 / dd : 1.0;
}
// inner matrix A D^-1 (column scaling)
template <typename T>
__global__ void batch_scale_kernel(int64_t nnz, const int* col, const double* A64, const double* dinv, T* A) {
    for (int64_t k = blockIdx.x * (int64_t)BS + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * BS)
        A[k] = (T)(A64[k] * dinv[col[k]]);
}
// per system: ||b||^2 and the initial state
__global__ void batch_init_kernel(int nprob, const int* prob_slice0, const int* prob_n, const double* b,
                                  BState* st) {
    __shared__ double sh[2 * MAX_BLOCK / 32];
    for (int pr = blockIdx.x; pr < nprob; pr += gridDim.x) {
        const int r0 = 32 * prob_slice0[pr], n = prob_n[pr];
        double a = 0.0, z = 0.0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) a += b[r0 + i] * b[r0 + i];
        blockSum2(a, z, sh);
        if (threadIdx.x == 0) {
            BState S{};
            S.bb = a;
            S.rho = S.alpha = S.omega = 1.0;
            S.state = a == 0.0 ? S_DONE : S_REFINE;  // b = 0: x = 0 (zeroed below)
            S.status = PRISM_OK;
            st[pr] = S;
        }
        __syncthreads();
    }
}
__global__ void batch_count_kernel(int nprob, const BState* st, int* ctl) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int a = 0;
    for (int p = 0; p < nprob; ++p) a += st[p].state == S_REFINE ? 1 : 0;
    ctl[0] = a;
    ctl[1] = a;
    ctl[2] = 0;
    ctl[3] = 0;
}
__global__ void zero_b0_kernel(int nprob, const int* prob_slice0, const int* prob_n, const BState* st, double* x) {
    for (int pr = blockIdx.x; pr < nprob; pr += gridDim.x) {
        if (st[pr].state != S_DONE) continue;
        const int r0 = 32 * prob_slice0[pr];
        for (int i = threadIdx.x; i < prob_n[pr]; i += blockDim.x) x[r0 + i] = 0.0;
    }
}

int smCountBatch() {
    static const int c = [] {
        int d = 0, v = 0;
        cudaGetDevice(&d);
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d);
        return v > 0 ? v : NUM_SMS;
    }();
    return c;
}

template <typename T>
void* kernelFor(int lpr) {
    if (lpr == 1) return (void*)batch_kernel<T, 1>;
    if (lpr == 2) return (void*)batch_kernel<T, 2>;
    return (void*)batch_kernel<T, 4>;
}

// All blocks co-resident (cooperative launch): one per slot the occupancy allows.
template <typename T>
void launchBatch(const BP<T>& P, int block, int lpr, cudaStream_t s) {
    void* fn = kernelFor<T>(lpr);
    const size_t smem = sizeof(int) * (2 * (size_t)P.nprob + 1 + 2 * (size_t)block + 2);
    if (smem > 48 * 1024) PB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    PB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, block, smem));
    if (per_sm < 1) fail(PRISM_INTERNAL, "batched solver: kernel does not fit on an SM");
    const int blocks = per_sm * smCountBatch();
    BP<T> args = P;
    void* kargs[] = {&args};
    PB_CUDA(cudaLaunchCooperativeKernel(fn, blocks, block, kargs, smem, s));
    countLaunch();
}

template <typename T>
struct InnerBufs {
    T* A;
    T *r, *r0, *p, *v, *s, *t, *d;
};
InnerBufs<float> innerBufs(BatchPlan& pl, float) {
    return {pl.A32f.p, pl.r32.p, pl.r032.p, pl.p32.p, pl.v32.p, pl.s32.p, pl.t32.p, pl.d32.p};
}
InnerBufs<double> innerBufs(BatchPlan& pl, double) {
    return {pl.A32d.p, pl.r64b.p, pl.r064.p, pl.p64.p, pl.v64.p, pl.s64.p, pl.t64.p, pl.d64.p};
}

template <typename T>
std::vector<BatchOut> runBatch(const std::vector<BatchSystem>& sys, BatchPlan& pl, double tol, double itol,
                               int max_inner, int max_pass, long long maxit, cudaStream_t s) {
    const int nrows = pl.nslices * 32;
    auto ensure = [&](auto& buf, size_t n) {
        if (buf.n != n) {
            buf.alloc(n);
            buf.zero(s);
        }
    };
    if constexpr (sizeof(T) == 4) {
        ensure(pl.A32f, pl.nnz);
        for (auto* b : {&pl.r32, &pl.r032, &pl.p32, &pl.v32, &pl.s32, &pl.t32, &pl.d32}) ensure(*b, nrows);
    } else {
        ensure(pl.A32d, pl.nnz);
        for (auto* b : {&pl.r64b, &pl.r064, &pl.p64, &pl.v64, &pl.s64, &pl.t64, &pl.d64}) ensure(*b, nrows);
    }
    InnerBufs<T> ib = innerBufs(pl, T{});
    // the systems' buffers, for the gather and scatter kernels (one grid row per system)
    if (sys.size() > 65535) fail(PRISM_BAD_ARG, "batched solve: at most 65535 systems per call");
    std::vector<CopyEntry> tab(sys.size());
    for (size_t i = 0; i < sys.size(); ++i) {
        const BatchSystem& q = sys[i];
        tab[i] = {q.vals, q.b, q.x, (long long)q.nnz_padded, (long long)pl.nnz_off[i], 32LL * pl.slice0[i], q.n};
    }
    std::vector<uintptr_t> key = {sizeof(T), (uintptr_t)max_inner, (uintptr_t)max_pass, (uintptr_t)maxit};
    for (double v : {tol, itol}) {
        uint64_t bits;
        std::memcpy(&bits, &v, sizeof bits);
        key.push_back((uintptr_t)bits);
    }
    for (const auto& e : tab)
        for (uintptr_t v : {(uintptr_t)e.vals, (uintptr_t)e.b, (uintptr_t)e.x}) key.push_back(v);
    const size_t tab_bytes = tab.size() * sizeof(CopyEntry);
    // graph_key = this prefix (6 entries) + the systems' pointers + the launch shape (2 entries)
    const bool same_systems = pl.graph_key.size() == key.size() + 2 &&
                              std::equal(key.begin() + 6, key.end(), pl.graph_key.begin() + 6);
    if (!same_systems) {
        if (pl.copy_tab.n < tab_bytes) pl.copy_tab.alloc(tab_bytes);
        pl.copy_tab.upload(reinterpret_cast<const unsigned char*>(tab.data()), tab_bytes, s);
    }
    const CopyEntry* dtab = reinterpret_cast<const CopyEntry*>(pl.copy_tab.p);
    const dim3 copy_grid(64, (unsigned)sys.size());
    auto gather = [&] {
        batch_copy_kernel<<<copy_grid, BS, 0, s>>>(dtab, 0, pl.A64.p, pl.b64.p, pl.x64.p); countLaunch();
        batch_dinv_kernel<<<grid(nrows), BS, 0, s>>>(nrows, pl.diag.p, pl.A64.p, pl.dinv.p); countLaunch();
        const int sg = (int)std::min<int64_t>(grid(pl.nnz), NUM_SMS * 32);
        batch_scale_kernel<T><<<sg, BS, 0, s>>>(pl.nnz, pl.col.p, pl.A64.p, pl.dinv.p, ib.A); countLaunch();
        PB_LAUNCH("batched setup");
    };

    BP<T> P{};
    P.nprob = pl.nprob;
    P.nslices = pl.nslices;
    P.slice_prob = pl.slice_prob.p;
    P.prob_slice0 = pl.prob_slice0.p;
    P.prob_n = pl.prob_n.p;
    P.sl_off = pl.sl_off.p;
    P.col = pl.col.p;
    P.A64 = pl.A64.p;
    P.A = ib.A;
    P.b64 = pl.b64.p;
    P.dinv = pl.dinv.p;
    P.x64 = pl.x64.p;
    P.r = ib.r;
    P.r0 = ib.r0;
    P.p = ib.p;
    P.v = ib.v;
    P.s = ib.s;
    P.t = ib.t;
    P.d = ib.d;
    P.cdot = pl.cdot.p;
    P.sdot = pl.cdot.p + 3 * (int64_t)pl.nslices * 4;
    P.st = reinterpret_cast<BState*>(pl.state.p);
    P.ctl = pl.ctl.p;
    P.tol2 = tol * tol;
    P.itol2 = itol * itol;
    P.max_inner = max_inner;
    P.max_pass = max_pass;
    P.maxit = maxit;

    auto init = [&] {
        PB_CUDA(cudaMemsetAsync(ib.d, 0, nrows * sizeof(T), s));
        batch_init_kernel<<<std::min(pl.nprob, NUM_SMS * 4), BS, 0, s>>>(pl.nprob, pl.prob_slice0.p, pl.prob_n.p,
                                                                         pl.b64.p, P.st); countLaunch();
        zero_b0_kernel<<<std::min(pl.nprob, NUM_SMS * 4), BS, 0, s>>>(pl.nprob, pl.prob_slice0.p, pl.prob_n.p, P.st,
                                                                      pl.x64.p); countLaunch();
        batch_count_kernel<<<1, 32, 0, s>>>(pl.nprob, P.st, P.ctl); countLaunch();
        PB_LAUNCH("batched init");
    };
    // autotune the launch shape on this batch: a few steps of every candidate from the same start
    BatchTuning& tune = pl.tune[sizeof(T) == 4 ? 1 : 0];
    if (tune.block == 0) {
        gather();
        DevBuf<double> xsave(nrows);
        PB_CUDA(cudaMemcpyAsync(xsave.p, pl.x64.p, nrows * sizeof(double), cudaMemcpyDeviceToDevice, s));
        cudaEvent_t e0, e1;
        PB_CUDA(cudaEventCreate(&e0));
        PB_CUDA(cudaEventCreate(&e1));
        for (int block : {128, 256, 512}) {
            for (int lpr : {1, 2, 4}) {
                init();
                BP<T> Q = P;
                Q.max_steps = 8;
                PB_CUDA(cudaEventRecord(e0, s));
                launchBatch(Q, block, lpr, s);
                PB_CUDA(cudaEventRecord(e1, s));
                PB_CUDA(cudaEventSynchronize(e1));
                float ms = 0.f;
                PB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                if (tune.block == 0 || ms < tune.ms) {
                    tune.block = block;
                    tune.lpr = lpr;
                    tune.ms = ms;
                }
                PB_CUDA(cudaMemcpyAsync(pl.x64.p, xsave.p, nrows * sizeof(double), cudaMemcpyDeviceToDevice, s));
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (verbose())
            std::fprintf(stderr, "[prism] batched solver tuned: block %d, %d lanes per row (%.3f ms for 8 steps)\n",
                         tune.block, tune.lpr, tune.ms);
    }
    // every step is one iteration (plus at most one refinement) of every active system
    P.max_steps = (int)std::min<long long>(maxit + (long long)max_pass + 2, (long long)1 << 30);
    key.push_back((uintptr_t)tune.block);
    key.push_back((uintptr_t)tune.lpr);
    // the call: gather, set-up, the persistent solve and the scatter of the solutions
    auto call = [&] {
        gather();
        init();
        launchBatch(P, tune.block, tune.lpr, s);
        PB_LAUNCH("batched solve");
        batch_copy_kernel<<<copy_grid, BS, 0, s>>>(dtab, 1, pl.A64.p, pl.b64.p, pl.x64.p); countLaunch();
    };
    const auto t0 = std::chrono::steady_clock::now();
    if (pl.graph.g && key == pl.graph_key) {
        PB_CUDA(cudaGraphLaunch(pl.graph.g, s));
        graphLaunchCounter().fetch_add(1, std::memory_order_relaxed);
    } else {
        pl.graph.reset();
        pl.graph_key.clear();
        // a capture that the runtime refuses leaves nothing executed: run the call directly
        cudaGraph_t g = nullptr;
        bool captured = false;
        if (cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed) == cudaSuccess) {
            try {
                call();
                captured = cudaStreamEndCapture(s, &g) == cudaSuccess && g != nullptr;
            } catch (...) {
                cudaStreamEndCapture(s, &g);
            }
            if (captured && cudaGraphInstantiate(&pl.graph.g, g, 0) != cudaSuccess) {
                pl.graph.g = nullptr;
                captured = false;
            }
            if (g) cudaGraphDestroy(g);
        }
        cudaGetLastError();
        if (captured) {
            pl.graph_key = key;
            PB_CUDA(cudaGraphLaunch(pl.graph.g, s));
            graphLaunchCounter().fetch_add(1, std::memory_order_relaxed);
        } else {
            call();
        }
    }
    if (verbose()) {
        PB_CUDA(cudaStreamSynchronize(s));
        std::fprintf(stderr, "[prism] batched solve of %d systems (%d rows): %.3f ms in one graph launch\n", pl.nprob,
                     nrows, std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    }
    std::vector<BState> hs(pl.nprob);
    PB_CUDA(cudaMemcpyAsync(hs.data(), P.st, pl.nprob * sizeof(BState), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
    std::vector<BatchOut> out(pl.nprob);
    for (int i = 0; i < pl.nprob; ++i) {
        out[i].iterations = hs[i].iter;
        out[i].passes = hs[i].pass;
        out[i].rel_residual = hs[i].bb > 0 ? std::sqrt(hs[i].rr64 / hs[i].bb) : 0.0;
        out[i].status = hs[i].state == S_DONE ? PRISM_OK
                                              : (hs[i].status != PRISM_OK ? hs[i].status : PRISM_NOT_CONVERGED);
    }
    return out;
}

}  // namespace

std::vector<BatchOut> solveBatch(const std::vector<BatchSystem>& sys, BatchPlan& pl, bool mixed, double tol,
                                 double itol, int max_inner, int max_pass, long long maxit, cudaStream_t s) {
    if (sys.empty()) return {};
    std::vector<uintptr_t> key;
    for (const auto& q : sys) {
        key.push_back((uintptr_t)q.sl_off);
        key.push_back((uintptr_t)q.sl_col);
        key.push_back((uintptr_t)q.n);
        key.push_back((uintptr_t)q.nnz_padded);
    }
    if (key != pl.key) {
        BatchPlan fresh;
        pl = std::move(fresh);
        pl.key = key;
        pl.nprob = (int)sys.size();
        std::vector<int> prob_slice0(pl.nprob + 1), prob_n(pl.nprob);
        pl.nnz_off.resize(pl.nprob + 1);
        pl.slice0.resize(pl.nprob + 1);
        int64_t nnz = 0;
        int64_t ns = 0;
        for (int i = 0; i < pl.nprob; ++i) {
            pl.nnz_off[i] = nnz;
            pl.slice0[i] = (int)ns;
            prob_slice0[i] = (int)ns;
            prob_n[i] = sys[i].n;
            nnz += sys[i].nnz_padded;
            ns += sys[i].nslices;
        }
        if (nnz >= ((int64_t)1 << 31) || ns * 32 >= ((int64_t)1 << 31) / 4)
            fail(PRISM_BAD_ARG, "batched solver: batch too large for 32-bit indices");
        if (pl.nprob > 16384) fail(PRISM_BAD_ARG, "batched solver: at most 16384 systems per batch");
        pl.nnz_off[pl.nprob] = nnz;
        pl.slice0[pl.nprob] = (int)ns;
        prob_slice0[pl.nprob] = (int)ns;
        pl.nnz = nnz;
        pl.nslices = (int)ns;
        const int nrows = pl.nslices * 32;
        pl.prob_slice0.upload(prob_slice0, s);
        pl.prob_n.upload(prob_n, s);
        pl.slice_prob.alloc(ns);
        pl.sl_off.alloc(ns + 1);
        pl.col.alloc(std::max<int64_t>(nnz, 1));
        pl.diag.alloc(nrows);
        fill_int_kernel<<<grid(nrows), BS, 0, s>>>(nrows, -1, pl.diag.p); countLaunch();
        for (int i = 0; i < pl.nprob; ++i) {
            const BatchSystem& q = sys[i];
            fill_int_kernel<<<grid(q.nslices), BS, 0, s>>>(q.nslices, i, pl.slice_prob.p + pl.slice0[i]); countLaunch();
            shift_kernel<<<grid(q.nslices), BS, 0, s>>>(q.nslices, q.sl_off, (int)pl.nnz_off[i],
                                                        pl.sl_off.p + pl.slice0[i]); countLaunch();
            const int gs = (int)std::min<int64_t>(grid(q.nnz_padded), NUM_SMS * 8);
            shift_kernel<<<gs, BS, 0, s>>>(q.nnz_padded, q.sl_col, 32 * pl.slice0[i], pl.col.p + pl.nnz_off[i]); countLaunch();
            shift_kernel<<<grid(q.n), BS, 0, s>>>(q.n, q.diag_pos, (int)pl.nnz_off[i],
                                                  pl.diag.p + 32 * (int64_t)pl.slice0[i]); countLaunch();
        }
        const int last = (int)nnz;
        PB_CUDA(cudaMemcpyAsync(pl.sl_off.p + ns, &last, sizeof(int), cudaMemcpyHostToDevice, s));
        pl.A64.alloc(std::max<int64_t>(nnz, 1));
        for (auto* b : {&pl.x64, &pl.b64, &pl.dinv}) {
            b->alloc(nrows);
            b->zero(s);
        }
        pl.cdot.alloc((size_t)ns * 4 * 3 + (size_t)ns * 2);
        pl.state.alloc(sizeof(BState) * pl.nprob);
        pl.ctl.alloc(4);
        PB_CUDA(cudaStreamSynchronize(s));
        PB_LAUNCH("batched plan");
    }
    if (mixed) return runBatch<float>(sys, pl, tol, itol, max_inner, max_pass, maxit, s);
    return runBatch<double>(sys, pl, tol, itol, max_inner, max_pass, maxit, s);
}

}  // namespace pb
