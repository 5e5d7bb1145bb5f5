// assemble.cu -- fused face-loop assembly of one eqn::Transport.
//
// One thread owns one matrix row (cell). It walks the cell's faces in the
// reference's insertion order (boundary faces patch by patch as
// applyBoundary visits them, then interior faces by face id as
// IFullScheme::apply visits them, scheme.cpp:12-22) and evaluates, for its own
// row only, every scheme of the equation:
//   convection  IConvection::applyInterior + Upwind::interpolate + weightsNVF
//               (convection.cpp:18-128, convection_hr.cpp:6-23) and the
//               Fixed/Outlet/ZeroGradient handlers (convection_boundary.cpp:4-61);
//   diffusion   NonCorrected / Corrected (diffusion.h:116-205) with the
//               over-relaxed / minimum / orthogonal decomposition
//               (nonortho.cpp:7-21) and Fixed/NoSlip/FixedGradient handlers
//               (diffusion_boundary.h:113-234);
//   sources     ConstantScalar / Divergence / Gradient (scheme/source/*.h);
//   symmetry    eqn::boundary::Symmetry<Transport> (equation/symmetry.cpp:54-90).
// Per-scheme partial sums are kept apart and combined in Transport::updateCoeffs
// order (transport.cpp:4-21), so with FMA contraction disabled the result is
// the reference's arithmetic, term for term. Each interior face is evaluated
// by both of its cells; no value is written by two threads and no atomics are
// used, so assembly is deterministic.
#include "assemble.h"
#include "devmath.cuh"

namespace pb {

struct NVF {
    double l, k;
};
// weightsNVF (convection.cpp:69-128); SMART keeps 1/6 == 5/6 == 3/8 == 0 (integer division)
__device__ __forceinline__ NVF weightsNVF(int scheme, double t) {
    switch (scheme) {
        case PRISM_CONV_CENTRAL: return {0.5, 0.5};
        case PRISM_CONV_LINEAR_UPWIND: return {1.5, 0.0};
        case PRISM_CONV_QUICK: return {0.75, 3.0 / 8.0};
        case PRISM_CONV_FROMM: return {1.0, 0.25};
        case PRISM_CONV_MINMOD:
            if (t > 0.0 && t < 0.5) return {1.5, 0.0};
            if (t >= 0.5 && t < 1.0) return {0.5, 0.5};
            return {1.0, 0.0};
        case PRISM_CONV_MUSCL:
            if (t > 0.0 && t < 0.25) return {2.0, 0.0};
            if (t >= 0.25 && t < 0.75) return {1.0, 0.25};
            if (t >= 0.75 && t < 1.0) return {0.0, 1.0};
            return {1.0, 0.0};
        case PRISM_CONV_SMART:
            if (t > 0.0 && t < 0.0) return {4.0, 0.0};
            if (t >= 0.0 && t < 0.0) return {0.75, 0.0};
            if (t >= 0.0 && t < 1.0) return {0.0, 1.0};
            return {1.0, 0.0};
        default: return {1.0, 0.0};
    }
}

// Upwind::interpolate for the row of `c` across a face to `n` with flux m_dot
// leaving c (convection.cpp:46-67).
__device__ __forceinline__ void interpolate(int scheme, double m_dot, double phi_c, double phi_n, D3 g_c, D3 g_n,
                                            D3 x_c, D3 x_n, double& aC, double& aN, double& b) {
    double pu = phi_n - (2 * dot(g_c, x_n - x_c));
    double t = (phi_c - pu) / (phi_n - pu);
    NVF w = weightsNVF(scheme, t);
    aC = smax(m_dot, 0.0) * w.l;
    aN = smax(m_dot, 0.0) * w.k;
    b = -smax(m_dot, 0.0) * (1 - w.l - w.k) * pu;
    double pu2 = phi_c - (2 * dot(g_n, x_c - x_n));
    double t2 = (phi_n - pu2) / (phi_c - pu2);
    NVF w2 = weightsNVF(scheme, t2);
    aC += -smax(-m_dot, 0.0) * w2.k;
    aN += -smax(-m_dot, 0.0) * w2.l;
    b += smax(-m_dot, 0.0) * (1 - w2.l - w2.k) * pu2;
}

__device__ __forceinline__ D3 kappaFace(const AssembleParams& P, int f, D3 v) {
    if (P.diff.kappa_tensor) return tensorTmulFace(P.m, P.diff.kt, f, v);
    return scalarFace(P.m, P.diff.ks, f) * v;
}
__device__ __forceinline__ D3 kappaCell(const AssembleParams& P, int c, D3 v) {
    if (P.diff.kappa_tensor) return tensorTmulCell(P.diff.kt, c, v);
    return P.diff.ks.v[c] * v;
}
__device__ __forceinline__ void decompose(int corr, D3 S, D3 e, D3& E, D3& T) {
    if (corr == PRISM_CORR_OVER_RELAXED) E = (dot(S, S) / (dot(e, S) + EPSILON)) * e;
    else if (corr == PRISM_CORR_MINIMUM) E = dot(e, S) * e;
    else E = norm(S) * e;
    T = S - E;
}

__global__ void __launch_bounds__(256) assemble_kernel(const AssembleParams P) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const MeshView& m = P.m;
    if (c >= m.nc) return;
    const ScalarView& phi = P.phi;
    const D3 xc = cellCenter(m, c);
    const double phic = phi.v[c];
    D3 gradc{0, 0, 0};
    if (P.need_grad) gradc = gradAt(phi, c);

    double dcv = 0.0, ddf = 0.0, rcv = 0.0, rdf = 0.0;
    // symmetry handler sums, one per patch, applied in patch order after the sources
    double sym_a[6], sym_b[6];
    int nsym = 0, sym_patch = -1;

    // zero this row's coefficients when the equation is clean
    const int slice = c >> 5, lane = c & 31;
    const int rb = m.sl_off[slice], width = (m.sl_off[slice + 1] - rb) >> 5;
    if (!P.accumulate)
        for (int j = 0; j < width; ++j) P.A[rb + 32 * j + lane] = 0.0;

    for (int q = P.ca_off[c]; q < P.ca_off[c + 1]; ++q) {
        const int f = P.ca_face[q];
        if (f < m.nb) {
            const int p = m.bpatch[f];
            if (m.patch_empty[p]) continue;
            const int k = phi.bc_kind[p];
            const D3 Sf = areaVector(m, f);
            if (P.has_conv) {
                if (k == PRISM_BC_FIXED) {
                    double phi_wall = phi.bc_val[p];
                    double mdot = vectorFlux(m, P.conv.U, f);
                    dcv += smax(mdot, 0.0);
                    rcv += smax(-mdot, 0.0) * phi_wall;
                } else if (k == PRISM_BC_OUTLET || k == PRISM_BC_ZERO_GRADIENT) {
                    D3 Uf = vectorFace(m, P.conv.U, f);
                    dcv += dot(Uf, Sf);
                }
            }
            if (P.has_diff) {
                if (k == PRISM_BC_FIXED || k == PRISM_BC_NOSLIP) {
                    double phi_wall = scalarFace(m, phi, f);
                    D3 d_Cf = faceCenter(m, f) - xc;
                    double dn = norm(d_Cf);
                    D3 Sp = kappaCell(P, c, Sf);
                    if (!P.diff.corrected) {
                        double g = dot(Sp, d_Cf) / (dn * dn + EPSILON);
                        ddf += g;
                        rdf += g * phi_wall;
                    } else {
                        D3 e = d_Cf / dn;
                        D3 E, T;
                        decompose(P.diff.corrector, Sp, e, E, T);
                        double g = dot(E, d_Cf) / (dn * dn + EPSILON);
                        ddf += g;
                        rdf += (g * phi_wall) + dot(T, gradFace(m, phi, f));
                    }
                } else if (k == PRISM_BC_FIXED_GRADIENT) {
                    D3 wg{phi.bc_vec[3 * p], phi.bc_vec[3 * p + 1], phi.bc_vec[3 * p + 2]};
                    D3 Sp = kappaCell(P, c, Sf);
                    rdf += -dot(wg, Sp);
                }
            }
            if (P.symmetry && k == PRISM_BC_SYMMETRY) {
                D3 n = faceNormal(m, f);
                double d_normal = dot(faceCenter(m, f) - xc, n);
                const VectorView& U = P.conv.U;
                D3 Uc{U.c[0].v[c], U.c[1].v[c], U.c[2].v[c]};
                double g = 2 * norm(kappaCell(P, c, Sf)) / d_normal;
                double ac, bb;
                if (P.phi_coord == 0) {
                    ac = n.x * n.x;
                    bb = ((Uc.y * n.y) + (Uc.z * n.z)) * n.x;
                } else if (P.phi_coord == 1) {
                    ac = n.y * n.y;
                    bb = ((Uc.x * n.x) + (Uc.z * n.z)) * n.y;
                } else {
                    ac = n.z * n.z;
                    bb = ((Uc.x * n.x) + (Uc.y * n.y)) * n.z;
                }
                if (p != sym_patch) {
                    sym_patch = p;
                    sym_a[nsym] = 0.0;
                    sym_b[nsym] = 0.0;
                    ++nsym;
                }
                sym_a[nsym - 1] += g * ac;
                sym_b[nsym - 1] += -g * bb;
            }
        } else {
            const int o = m.owner[f];
            const int nb_ = m.nbr[f];
            const bool own = (o == c);
            const int n = own ? nb_ : o;
            const D3 xn = cellCenter(m, n);
            double off_cv = 0.0, off_df = 0.0;
            if (P.has_conv) {
                double mdot = vectorFlux(m, P.conv.U, f);
                double aC, aN, b;
                interpolate(P.conv.scheme, own ? mdot : -mdot, phic, phi.v[n], gradc, gradAt(phi, n), xc, xn, aC, aN,
                            b);
                dcv += aC;
                off_cv = aN;
                rcv += b;
            }
            if (P.has_diff) {
                // owner-oriented quantities, so both cells compute the same g and T
                const D3 xo = own ? xc : xn, xnb = own ? xn : xc;
                const D3 d_CF = xnb - xo;
                const double dn = norm(d_CF);
                const D3 Sf = areaVector(m, f);
                double g;
                if (!P.diff.corrected) {
                    D3 Sp = kappaFace(P, f, Sf);
                    g = dot(Sp, d_CF) / (dn * dn + EPSILON);
                } else {
                    D3 e = d_CF / dn;
                    D3 Sp = kappaFace(P, f, Sf);
                    D3 E, T;
                    decompose(P.diff.corrector, Sp, e, E, T);
                    g = dot(E, d_CF) / (dn * dn + EPSILON);
                    D3 gf = gradFace(m, phi, f);
                    double t = dot(T, gf);
                    rdf += own ? t : -t;
                }
                ddf += g;
                off_df = -g;
            }
            const int pos = P.ca_pos[q];
            double a = P.accumulate ? P.A[pos] : 0.0;
            if (P.conv_first) {
                if (P.has_conv) a = a + off_cv;
                if (P.has_diff) a = a + off_df;
            } else {
                if (P.has_diff) a = a + off_df;
                if (P.has_conv) a = a + off_cv;
            }
            P.A[pos] = a;
        }
    }

    // sources (applied after the schemes, in registration order)
    double rsrc[MAX_SOURCES];
    for (int s = 0; s < P.nsrc; ++s) {
        const SourceDesc& S = P.src[s];
        double v;
        if (S.kind == PRISM_SRC_CONSTANT) {
            v = S.s.v[c] * m.vol[c];
        } else if (S.kind == PRISM_SRC_DIVERGENCE) {
            double d = fluxSum(m, S.U, c) / m.vol[c];
            v = d * m.vol[c];
        } else {
            v = S.s.g[S.coord * S.s.gstride + c] * m.vol[c];
        }
        rsrc[s] = S.sign == PRISM_SIGN_NEGATIVE ? -v : v;
    }

    // Transport::updateCoeffs: A += A_s, b += b_s per scheme (scheme rhs accumulates
    // across applies until zeroOutCoeffs), then sources, then equation handlers.
    const int dpos = m.diag_pos[c];
    double A = P.accumulate ? P.A[dpos] : 0.0;
    double b = P.accumulate ? P.b[c] : 0.0;
    double bcv = rcv, bdf = rdf;
    if (P.accumulate) {
        if (P.has_conv) bcv = P.bconv[c] + rcv;
        if (P.has_diff) bdf = P.bdiff[c] + rdf;
    }
    // temporal scheme (backward_euler.cpp:80-82, adam_moulton.cpp:94-98): diagonal and a
    // right-hand side assigned afresh on every apply
    double dtm = 0.0, btm = 0.0;
    if (P.has_temporal) {
        const double vol = m.vol[c];
        if (P.tm.second_order) {
            dtm = ((3.0 / 2.0) * vol) / P.tm.dt;
            btm = (2.0 * (vol * P.tm.prev[c])) / P.tm.dt;
            btm = btm + ((-0.5 * (vol * P.tm.prev2[c])) / P.tm.dt);
        } else {
            dtm = vol / P.tm.dt;
            btm = (vol * P.tm.prev[c]) / P.tm.dt;
        }
    }
    for (int k = 0; k < P.nsch; ++k) {
        const int kind = P.order[k];
        if (kind == SCH_CONV) {
            A = A + dcv;
            b = b + bcv;
        } else if (kind == SCH_DIFF) {
            A = A + ddf;
            b = b + bdf;
        } else {
            A = A + dtm;
            b = b + btm;
        }
    }
    for (int s = 0; s < P.nsrc; ++s) b = b + rsrc[s];
    for (int s = 0; s < nsym; ++s) {
        A = A + sym_a[s];
        b = b + sym_b[s];
    }
    P.A[dpos] = A;
    P.b[c] = b;
    if (P.has_conv) P.bconv[c] = bcv;
    if (P.has_diff) P.bdiff[c] = bdf;
}

void launchAssemble(const AssembleParams& P, cudaStream_t s) {
    if (P.m.nc == 0) return;
    assemble_kernel<<<ceil_div(P.m.nc, 256), 256, 0, s>>>(P); countLaunch();
    PB_LAUNCH("assemble_kernel");
}

// Transport::relax (transport.cpp:54-64)
__global__ void relax_kernel(double* A, double* b, const int* diag_pos, const double* phi, double alpha, int n) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    double d = A[diag_pos[c]];
    b[c] += ((1.0 - alpha) / alpha) * (d * phi[c]);
    A[diag_pos[c]] = d / alpha;
}
void launchRelax(double* A, double* b, const int* diag_pos, const double* phi, double alpha, int n, cudaStream_t s) {
    if (n == 0) return;
    relax_kernel<<<ceil_div(n, 256), 256, 0, s>>>(A, b, diag_pos, phi, alpha, n); countLaunch();
    PB_LAUNCH("relax_kernel");
}

// reference-cell pin (numerics/solver.cpp:50-57)
__global__ void pin_kernel(double* A, double* b, int pos, int row, double ref_value) {
    double diag = A[pos];
    A[pos] += diag;
    b[row] += diag * ref_value;
}
void launchPin(double* A, double* b, int pos, int row, double ref_value, cudaStream_t s) {
    pin_kernel<<<1, 1, 0, s>>>(A, b, pos, row, ref_value); countLaunch();
    PB_LAUNCH("pin_kernel");
}
// the same, with the diagonal's position read on the device (for graph capture)
__global__ void pin_dev_kernel(double* A, double* b, const int* diag_pos, int row, double ref_value) {
    const int pos = diag_pos[row];
    double diag = A[pos];
    A[pos] += diag;
    b[row] += diag * ref_value;
}
void launchPinDev(double* A, double* b, const int* diag_pos, int row, double ref_value, cudaStream_t s) {
    pin_dev_kernel<<<1, 1, 0, s>>>(A, b, diag_pos, row, ref_value); countLaunch();
    PB_LAUNCH("pin_dev_kernel");
}

}  // namespace pb
