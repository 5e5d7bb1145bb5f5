// adjoint.cu -- discrete adjoint of steady diffusion: transposed assembly terms.
//
// The converged state of repeated ISolver::solve calls on a diffusion equation
// (diffusion.h:116-205, diffusion_boundary.h:113-234, least-squares gradient
// least_squares.cpp:63-100) satisfies R(phi, kappa, v) = A phi - b = 0, where b
// holds the explicit non-orthogonal correction T_f . grad(phi)_f and the
// Dirichlet face values v. R is linear in phi:
//   R = A phi - C phi - b0,   C phi = correction terms through G phi (G: the
//   least-squares gradient operator) and the boundary-face gradient.
// For J(phi) the adjoint lambda solves (A - C)^T lambda = dJ/dphi. It is
// computed by the transposed deferred correction the forward uses,
//   A^T lambda_{k+1} = dJ/dphi + C^T lambda_k,
// one transposed BiCGSTAB solve per step (A^T assembled by permuting A's
// values), so no Krylov history is stored: every step recomputes C^T lambda
// from the mesh, kappa and lambda. Then
//   dJ/dkappa_c = -lambda^T dR/dkappa_c,   dJ/dv_f = -lambda^T dR/dv_f.
// All kernels are cell-owned gathers (no atomics); each boundary face is
// written by its owner cell only.
#include "adjoint.h"
#include "devmath.cuh"

namespace pb {

namespace {

constexpr int BS = 256;
inline int grid(int64_t n) { return std::max(1, ceil_div(n, BS)); }

// g and T of one face for a scalar coefficient kappa (S' = kappa S), and their
// derivatives in kappa, with the expressions of the assembly kernel.
struct DiffFace {
    double g, dg;
    D3 T, dT;
};
__device__ __forceinline__ DiffFace diffFace(int corrected, int corr, double kappa, D3 S, D3 d) {
    DiffFace r;
    const double dn = norm(d);
    const double den = dn * dn + EPSILON;
    const D3 Sp = kappa * S;
    if (!corrected) {
        r.g = dot(Sp, d) / den;
        r.dg = dot(S, d) / den;
        r.T = d3(0, 0, 0);
        r.dT = d3(0, 0, 0);
        return r;
    }
    const D3 e = d / dn;
    D3 E, dE;
    if (corr == PRISM_CORR_OVER_RELAXED) {
        const double a = dot(Sp, Sp), b = dot(e, Sp) + EPSILON;
        E = (a / b) * e;
        // a = kappa^2 |S|^2, b = kappa e.S + eps
        dE = ((2.0 * kappa * dot(S, S) * b - a * dot(e, S)) / (b * b)) * e;
    } else if (corr == PRISM_CORR_MINIMUM) {
        E = dot(e, Sp) * e;
        dE = dot(e, S) * e;
    } else {
        E = norm(Sp) * e;
        dE = (kappa >= 0.0 ? norm(S) : -norm(S)) * e;
    }
    r.T = Sp - E;
    r.dT = S - dE;
    r.g = dot(E, d) / den;
    r.dg = dot(dE, d) / den;
    return r;
}

__device__ __forceinline__ D3 lsWeight(const AdjointParams& P, int q) {
    return d3(P.w[q], P.w[P.nk + q], P.w[2 * P.nk + q]);
}
__device__ __forceinline__ D3 load3(const double* u, int64_t stride, int c) {
    return d3(u[c], u[stride + c], u[2 * stride + c]);
}
// the least-squares "other" value of boundary face f does not follow phi_c
__device__ __forceinline__ bool boundaryValueFixed(const ScalarView& s, int k) {
    return s.fv != nullptr || k == PRISM_BC_FIXED || k == PRISM_BC_NOSLIP;
}

__global__ void twin_kernel(const MeshView m, int* twin) {
    int c = blockIdx.x * BS + threadIdx.x;
    if (c >= m.nc) return;
    for (int q = m.cf_off[c]; q < m.cf_off[c + 1]; ++q) {
        const int f = m.cf_face[q];
        int t = -1;
        if (f >= m.nb) {
            const int o = m.owner[f];
            const int other = (o == c) ? m.nbr[f] : o;
            for (int p = m.cf_off[other]; p < m.cf_off[other + 1]; ++p)
                if (m.cf_face[p] == f) t = p;
        }
        twin[q] = t;
    }
}

__global__ void tpos_kernel(int n, int nslices, const int* rowptr, const int* sl_off, const int* sl_col, int* tpos) {
    int r = blockIdx.x * BS + threadIdx.x;
    if (r >= nslices * 32) return;
    const int s = r >> 5, lane = r & 31;
    const int base = sl_off[s], width = (sl_off[s + 1] - base) >> 5;
    const int len = r < n ? rowptr[r + 1] - rowptr[r] : 0;
    for (int j = 0; j < width; ++j) {
        const int pos = base + 32 * j + lane;
        int t = pos;  // padding: its own (zero) slot
        if (j < len) {
            const int c = sl_col[pos];
            const int cb = sl_off[c >> 5] + (c & 31);
            const int clen = rowptr[c + 1] - rowptr[c];
            for (int i = 0; i < clen; ++i)
                if (sl_col[cb + 32 * i] == r) t = cb + 32 * i;
        }
        tpos[pos] = t;
    }
}

__global__ void transpose_values_kernel(int64_t nnz, const int* tpos, const double* A, double* AT) {
    for (int64_t k = blockIdx.x * (int64_t)BS + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * BS) AT[k] = A[tpos[k]];
}

// psi_c = sum_int (l_N - l_O) w_c T_f - sum_Dirichlet l_c (T_b - (T_b.e) e);  u_c = pinv_c^T psi_c;
// d_c = sum_Dirichlet (T_b.e) / |d_Cf|
__global__ void __launch_bounds__(BS) correction_kernel(const AdjointParams P, const double* __restrict__ lam,
                                                        double* __restrict__ u, double* __restrict__ d,
                                                        int64_t stride) {
    const int c = blockIdx.x * BS + threadIdx.x;
    const MeshView& m = P.m;
    if (c >= m.nc) return;
    D3 psi{0, 0, 0};
    double dsum = 0.0;
    if (P.corrected) {
        const D3 xc = cellCenter(m, c);
        const double lc = lam[c];
        for (int q = m.cf_off[c]; q < m.cf_off[c + 1]; ++q) {
            const int f = m.cf_face[q];
            const D3 Sf = areaVector(m, f);
            if (f < m.nb) {
                const int p = m.bpatch[f];
                if (m.patch_empty[p]) continue;
                const int k = P.phi.bc_kind[p];
                if (k != PRISM_BC_FIXED && k != PRISM_BC_NOSLIP) continue;
                const D3 dCf = faceCenter(m, f) - xc;
                const double dn = norm(dCf);
                const D3 e = dCf / dn;
                const DiffFace F = diffFace(1, P.corrector, P.ks.v[c], Sf, dCf);
                const double te = dot(F.T, e);
                psi = psi - lc * (F.T - te * e);
                dsum += te / dn;
            } else {
                const int o = m.owner[f], nn = m.nbr[f];
                const D3 dCF = cellCenter(m, nn) - cellCenter(m, o);
                const DiffFace F = diffFace(1, P.corrector, scalarFace(m, P.ks, f), Sf, dCF);
                const double gcw = m.gcw[f - m.nb];
                const double wc = (o == c) ? gcw : 1.0 - gcw;
                psi = psi + ((lam[nn] - lam[o]) * wc) * F.T;
            }
        }
    }
    const int64_t n = m.nc;
    D3 uc;
    uc.x = (P.pinv[0 * n + c] * psi.x + P.pinv[3 * n + c] * psi.y) + P.pinv[6 * n + c] * psi.z;
    uc.y = (P.pinv[1 * n + c] * psi.x + P.pinv[4 * n + c] * psi.y) + P.pinv[7 * n + c] * psi.z;
    uc.z = (P.pinv[2 * n + c] * psi.x + P.pinv[5 * n + c] * psi.y) + P.pinv[8 * n + c] * psi.z;
    u[c] = uc.x;
    u[stride + c] = uc.y;
    u[2 * stride + c] = uc.z;
    d[c] = dsum;
}

// rhs_k = dJ_k - (G^T psi)_k - d_k lambda_k
__global__ void __launch_bounds__(BS) rhs_kernel(const AdjointParams P, const double* __restrict__ dJ,
                                                 const double* __restrict__ lam, const double* __restrict__ u,
                                                 const double* __restrict__ d, int64_t stride,
                                                 double* __restrict__ rhs) {
    const int k = blockIdx.x * BS + threadIdx.x;
    const MeshView& m = P.m;
    if (k >= m.nc) return;
    double acc = 0.0;
    if (P.corrected) {
        const D3 uk = load3(u, stride, k);
        for (int q = m.cf_off[k]; q < m.cf_off[k + 1]; ++q) {
            const int f = m.cf_face[q];
            if (f < m.nb) {
                const int p = m.bpatch[f];
                if (m.patch_empty[p]) continue;
                if (boundaryValueFixed(P.phi, P.phi.bc_kind[p])) acc -= dot(uk, lsWeight(P, q));
            } else {
                const int o = m.owner[f];
                const int c = (o == k) ? m.nbr[f] : o;
                acc += dot(load3(u, stride, c), lsWeight(P, P.twin[q])) - dot(uk, lsWeight(P, q));
            }
        }
    }
    rhs[k] = dJ[k] - acc - d[k] * lam[k];
}

__global__ void __launch_bounds__(BS) gradients_kernel(const AdjointParams P, const double* __restrict__ lam,
                                                       const double* __restrict__ u, int64_t stride,
                                                       double* __restrict__ gk, double* __restrict__ gv) {
    const int c = blockIdx.x * BS + threadIdx.x;
    const MeshView& m = P.m;
    if (c >= m.nc) return;
    const D3 xc = cellCenter(m, c);
    const double lc = lam[c], phic = P.phi.v[c];
    const D3 uc = load3(u, stride, c);
    double g = 0.0;
    for (int q = m.cf_off[c]; q < m.cf_off[c + 1]; ++q) {
        const int f = m.cf_face[q];
        const D3 Sf = areaVector(m, f);
        if (f < m.nb) {
            const int p = m.bpatch[f];
            if (m.patch_empty[p]) continue;
            const int k = P.phi.bc_kind[p];
            double gvf = 0.0;
            if (k == PRISM_BC_FIXED || k == PRISM_BC_NOSLIP) {
                const double wall = scalarFace(m, P.phi, f);
                const D3 dCf = faceCenter(m, f) - xc;
                const double dn = norm(dCf);
                const DiffFace F = diffFace(P.corrected, P.corrector, P.ks.v[c], Sf, dCf);
                double dF = F.dg * (phic - wall);
                gvf = lc * F.g;
                if (P.corrected) {
                    dF -= dot(F.dT, gradFace(m, P.phi, f));
                    gvf += lc * dot(F.T, dCf / dn) / dn;
                }
                g -= lc * dF;
            } else if (k == PRISM_BC_FIXED_GRADIENT) {
                const D3 wg{P.phi.bc_vec[3 * p], P.phi.bc_vec[3 * p + 1], P.phi.bc_vec[3 * p + 2]};
                g -= lc * dot(wg, Sf);
            }
            if (P.corrected && boundaryValueFixed(P.phi, k)) gvf -= dot(uc, lsWeight(P, q));
            gv[f] = gvf;
        } else {
            const int o = m.owner[f], nn = m.nbr[f];
            const D3 dCF = cellCenter(m, nn) - cellCenter(m, o);
            const DiffFace F = diffFace(P.corrected, P.corrector, scalarFace(m, P.ks, f), Sf, dCF);
            double dF = F.dg * (P.phi.v[o] - P.phi.v[nn]);
            if (P.corrected) dF -= dot(F.dT, gradFace(m, P.phi, f));
            const double gcw = m.gcw[f - m.nb];
            const double dk = P.ks.fv ? 0.0 : ((o == c) ? gcw : 1.0 - gcw);
            g -= (lam[o] - lam[nn]) * dF * dk;
        }
    }
    gk[c] = g;
}

__global__ void __launch_bounds__(BS) diff_partials_kernel(int n, const double* a, const double* b, double* partials) {
    __shared__ double sh[2][BS / 32];
    double s0 = 0.0, s1 = 0.0;
    for (int i = blockIdx.x * BS + threadIdx.x; i < n; i += gridDim.x * BS) {
        const double x = a[i] - b[i];
        s0 += x * x;
        s1 += a[i] * a[i];
    }
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_down_sync(0xffffffffu, s0, o);
        s1 += __shfl_down_sync(0xffffffffu, s1, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sh[0][threadIdx.x >> 5] = s0;
        sh[1][threadIdx.x >> 5] = s1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0;
        for (int w = 0; w < BS / 32; ++w) {
            t0 += sh[0][w];
            t1 += sh[1][w];
        }
        partials[2 * blockIdx.x] = t0;
        partials[2 * blockIdx.x + 1] = t1;
    }
}
__global__ void diff_final_kernel(int nblocks, const double* partials, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double t0 = 0.0, t1 = 0.0;
    for (int b = 0; b < nblocks; ++b) {
        t0 += partials[2 * b];
        t1 += partials[2 * b + 1];
    }
    out[0] = t0;
    out[1] = t1;
}

}  // namespace

void buildTwin(const MeshView& m, int* twin, cudaStream_t s) {
    twin_kernel<<<grid(m.nc), BS, 0, s>>>(m, twin); countLaunch();
    PB_LAUNCH("twin_kernel");
}
void buildTransposePositions(int n, int nslices, const int* rowptr, const int* sl_off, const int* sl_col, int* tpos,
                             cudaStream_t s) {
    tpos_kernel<<<grid((int64_t)nslices * 32), BS, 0, s>>>(n, nslices, rowptr, sl_off, sl_col, tpos); countLaunch();
    PB_LAUNCH("tpos_kernel");
}
void transposeValues(int64_t nnz_padded, const int* tpos, const double* A, double* AT, cudaStream_t s) {
    const int g = (int)std::min<int64_t>(grid(nnz_padded), NUM_SMS * 32);
    transpose_values_kernel<<<g, BS, 0, s>>>(nnz_padded, tpos, A, AT); countLaunch();
    PB_LAUNCH("transpose_values_kernel");
}
void adjointCorrection(const AdjointParams& P, const double* lambda, double* u, double* d, int64_t stride,
                       cudaStream_t s) {
    correction_kernel<<<grid(P.m.nc), BS, 0, s>>>(P, lambda, u, d, stride); countLaunch();
    PB_LAUNCH("adjoint correction_kernel");
}
void adjointRhs(const AdjointParams& P, const double* dJ, const double* lambda, const double* u, const double* d,
                int64_t stride, double* rhs, cudaStream_t s) {
    rhs_kernel<<<grid(P.m.nc), BS, 0, s>>>(P, dJ, lambda, u, d, stride, rhs); countLaunch();
    PB_LAUNCH("adjoint rhs_kernel");
}
void adjointGradients(const AdjointParams& P, const double* lambda, const double* u, int64_t stride, double* gk,
                      double* gv, cudaStream_t s) {
    PB_CUDA(cudaMemsetAsync(gv, 0, std::max(P.m.nb, 1) * sizeof(double), s));
    gradients_kernel<<<grid(P.m.nc), BS, 0, s>>>(P, lambda, u, stride, gk, gv); countLaunch();
    PB_LAUNCH("adjoint gradients_kernel");
}
void diffNorms(int n, const double* a, const double* b, double* partials, unsigned int*, double* dev_out,
               double* host_out, cudaStream_t s) {
    const int nb = std::max(1, std::min(ceil_div(n, BS), NUM_SMS * 8));
    diff_partials_kernel<<<nb, BS, 0, s>>>(n, a, b, partials); countLaunch();
    diff_final_kernel<<<1, 32, 0, s>>>(nb, partials, dev_out); countLaunch();
    PB_LAUNCH("diff norms");
    PB_CUDA(cudaMemcpyAsync(host_out, dev_out, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace pb
