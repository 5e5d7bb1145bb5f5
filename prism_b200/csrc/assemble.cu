// assemble.cu -- face-loop assembly of one eqn::Transport in two passes.
//
// Face pass: one thread per non-empty face evaluates, once, every scheme term
// the face contributes to the rows of its cells:
//   convection  IConvection::applyInterior + Upwind::interpolate + weightsNVF
//               (convection.cpp:18-128, convection_hr.cpp:6-23) for the owner's
//               row and, with the flux reversed, the neighbour's (both from the
//               same pair of phi-tilde values) and the Fixed/Outlet/ZeroGradient
//               handlers (convection_boundary.cpp:4-61);
//   diffusion   NonCorrected / Corrected (diffusion.h:116-205) with the
//               over-relaxed / minimum / orthogonal decomposition
//               (nonortho.cpp:7-21) and the Fixed/NoSlip/FixedGradient handlers
//               (diffusion_boundary.h:113-234).
// It writes the off-diagonal coefficients (each interior face owns the two
// matrix entries it couples) and, per (cell, face) pair, a record of the terms
// that the cell's diagonal and right-hand side sum: convection diagonal, its
// rhs, diffusion diagonal, its rhs. The records sit in the cells' assembly-order
// lists, so the cell pass reads each cell's records contiguously.
// Cell pass: one thread per row sums its records in the reference's insertion
// order (boundary faces patch by patch as applyBoundary visits them, then
// interior faces by face id as IFullScheme::apply does, scheme.cpp:12-22),
// then the sources (scheme/source/*.h), the temporal term and the symmetry
// handler (equation/symmetry.cpp:54-90), and combines the per-scheme sums in
// Transport::updateCoeffs order (transport.cpp:4-21). With FMA contraction
// disabled the result is the reference's arithmetic, term for term; no value is
// written by two threads and no atomics are used, so assembly is deterministic.
// Empty-patch faces keep all-zero records: adding +0.0 to a sum that starts at
// +0.0 changes no bit. Padding slots of the SELL rows are never written (the
// matrix is zeroed on allocation and by zeroOutCoeffs).
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

__device__ __forceinline__ void putRec(double* rec, int q, double dc, double rc, double dd, double rd) {
    double4* r = reinterpret_cast<double4*>(rec) + q;
    *r = make_double4(dc, rc, dd, rd);
}

// at least 5 blocks of 256 per SM (48 registers, a few spilled to L1): 8% faster on the
// 128^3 transport assembly than 4 blocks at 64 registers
__global__ void __launch_bounds__(256, 5) assemble_faces_kernel(const AssembleParams P) {
    const MeshView& m = P.m;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.nne + (m.nf - m.nb)) return;
    const int f = i < m.nne ? i : m.nb + (i - m.nne);
    const ScalarView& phi = P.phi;
    if (f < m.nb) {
        // boundary face of a non-empty patch: terms of the owner's row
        const int c = m.owner[f];
        const int p = m.bpatch[f];
        const int k = phi.bc_kind[p];
        const D3 Sf = areaVector(m, f);
        double dc = 0.0, rc = 0.0, dd = 0.0, rd = 0.0;
        if (P.has_conv) {
            if (k == PRISM_BC_FIXED) {
                double phi_wall = phi.bc_val[p];
                double mdot = vectorFlux(m, P.conv.U, f);
                dc = smax(mdot, 0.0);
                rc = smax(-mdot, 0.0) * phi_wall;
            } else if (k == PRISM_BC_OUTLET || k == PRISM_BC_ZERO_GRADIENT) {
                D3 Uf = vectorFace(m, P.conv.U, f);
                dc = dot(Uf, Sf);
            }
        }
        if (P.has_diff) {
            if (k == PRISM_BC_FIXED || k == PRISM_BC_NOSLIP) {
                double phi_wall = scalarFace(m, phi, f);
                D3 d_Cf = faceCenter(m, f) - cellCenter(m, c);
                double dn = norm(d_Cf);
                D3 Sp = kappaCell(P, c, Sf);
                if (!P.diff.corrected) {
                    double g = dot(Sp, d_Cf) / (dn * dn + EPSILON);
                    dd = g;
                    rd = g * phi_wall;
                } else {
                    D3 e = d_Cf / dn;
                    D3 E, T;
                    decompose(P.diff.corrector, Sp, e, E, T);
                    double g = dot(E, d_Cf) / (dn * dn + EPSILON);
                    dd = g;
                    rd = (g * phi_wall) + dot(T, gradFace(m, phi, f));
                }
            } else if (k == PRISM_BC_FIXED_GRADIENT) {
                D3 wg{phi.bc_vec[3 * p], phi.bc_vec[3 * p + 1], phi.bc_vec[3 * p + 2]};
                D3 Sp = kappaCell(P, c, Sf);
                rd = -dot(wg, Sp);
            }
        }
        putRec(P.rec, P.face_slot[2 * f], dc, rc, dd, rd);
        return;
    }
    // interior face: owner o, neighbour n
    const int o = m.owner[f];
    const int n = m.nbr[f];
    const D3 xo = cellCenter(m, o), xn = cellCenter(m, n);
    double aCo = 0.0, aNo = 0.0, bo = 0.0, aCn = 0.0, aNn = 0.0, bn = 0.0;
    if (P.has_conv) {
        const double mdot = vectorFlux(m, P.conv.U, f);
        const double phio = phi.v[o], phin = phi.v[n];
        D3 go{0, 0, 0}, gn{0, 0, 0};
        if (P.need_grad) {
            go = gradAt(phi, o);
            gn = gradAt(phi, n);
        }
        // Upwind::interpolate from the owner's side (m_dot = mdot) and from the neighbour's
        // (m_dot = -mdot): the neighbour's phi-tilde pair is the owner's, swapped
        const double pu = phin - (2 * dot(go, xn - xo));
        const double t = (phio - pu) / (phin - pu);
        const NVF w = weightsNVF(P.conv.scheme, t);
        const double pu2 = phio - (2 * dot(gn, xo - xn));
        const double t2 = (phin - pu2) / (phio - pu2);
        const NVF w2 = weightsNVF(P.conv.scheme, t2);
        aCo = smax(mdot, 0.0) * w.l;
        aNo = smax(mdot, 0.0) * w.k;
        bo = -smax(mdot, 0.0) * (1 - w.l - w.k) * pu;
        aCo += -smax(-mdot, 0.0) * w2.k;
        aNo += -smax(-mdot, 0.0) * w2.l;
        bo += smax(-mdot, 0.0) * (1 - w2.l - w2.k) * pu2;
        const double mn = -mdot;
        aCn = smax(mn, 0.0) * w2.l;
        aNn = smax(mn, 0.0) * w2.k;
        bn = -smax(mn, 0.0) * (1 - w2.l - w2.k) * pu2;
        aCn += -smax(-mn, 0.0) * w.k;
        aNn += -smax(-mn, 0.0) * w.l;
        bn += smax(-mn, 0.0) * (1 - w.l - w.k) * pu;
    }
    double g = 0.0, tf = 0.0;
    if (P.has_diff) {
        const D3 d_CF = xn - xo;
        const double dn = norm(d_CF);
        const D3 Sf = areaVector(m, f);
        if (!P.diff.corrected) {
            D3 Sp = kappaFace(P, f, Sf);
            g = dot(Sp, d_CF) / (dn * dn + EPSILON);
        } else {
            D3 e = d_CF / dn;
            D3 Sp = kappaFace(P, f, Sf);
            D3 E, T;
            decompose(P.diff.corrector, Sp, e, E, T);
            g = dot(E, d_CF) / (dn * dn + EPSILON);
            tf = dot(T, gradFace(m, phi, f));
        }
    }
    // off-diagonal coefficients, the schemes' terms added in registration order
    const int pon = P.face_pos[2 * f], pno = P.face_pos[2 * f + 1];
    double a1 = P.accumulate ? P.A[pon] : 0.0;
    double a2 = P.accumulate ? P.A[pno] : 0.0;
    if (P.conv_first) {
        if (P.has_conv) {
            a1 = a1 + aNo;
            a2 = a2 + aNn;
        }
        if (P.has_diff) {
            a1 = a1 + -g;
            a2 = a2 + -g;
        }
    } else {
        if (P.has_diff) {
            a1 = a1 + -g;
            a2 = a2 + -g;
        }
        if (P.has_conv) {
            a1 = a1 + aNo;
            a2 = a2 + aNn;
        }
    }
    P.A[pon] = a1;
    P.A[pno] = a2;
    putRec(P.rec, P.face_slot[2 * f], aCo, bo, g, tf);
    putRec(P.rec, P.face_slot[2 * f + 1], aCn, bn, g, -tf);
}

__global__ void __launch_bounds__(256, 4) assemble_cells_kernel(const AssembleParams P) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const MeshView& m = P.m;
    if (c >= m.nc) return;

    // the rows' sums over the cell's faces, in insertion order
    double dcv = 0.0, ddf = 0.0, rcv = 0.0, rdf = 0.0;
    const double4* R = reinterpret_cast<const double4*>(P.rec);
    for (int q = P.ca_off[c]; q < P.ca_off[c + 1]; ++q) {
        const double4 r = R[q];
        dcv += r.x;
        rcv += r.y;
        ddf += r.z;
        rdf += r.w;
    }

    // symmetry handler sums, one per patch, applied in patch order after the sources
    double sym_a[6], sym_b[6];
    int nsym = 0, sym_patch = -1;
    if (P.symmetry) {
        const ScalarView& phi = P.phi;
        const D3 xc = cellCenter(m, c);
        for (int q = P.ca_off[c]; q < P.ca_off[c + 1]; ++q) {
            const int f = P.ca_face[q];
            if (f >= m.nb) continue;
            const int p = m.bpatch[f];
            if (m.patch_empty[p] || phi.bc_kind[p] != PRISM_BC_SYMMETRY) continue;
            const D3 Sf = areaVector(m, f);
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
    const int nfaces = P.m.nne + (P.m.nf - P.m.nb);
    if (nfaces > 0) {
        assemble_faces_kernel<<<ceil_div(nfaces, 256), 256, 0, s>>>(P); countLaunch();
        PB_LAUNCH("assemble_faces_kernel");
    }
    assemble_cells_kernel<<<ceil_div(P.m.nc, 256), 256, 0, s>>>(P); countLaunch();
    PB_LAUNCH("assemble_cells_kernel");
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
