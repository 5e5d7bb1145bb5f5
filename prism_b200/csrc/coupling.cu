// coupling.cu -- pressure-velocity coupling kernels of the SIMPLE / PRIME drivers.
//
//   d_tensor      pressureEquationCoeffsTensor (algorithm/SIMPLE.cpp:77-108):
//                 D = diag(V/(a_P^u+eps), V/(a_P^v+eps), V/(a_P^w+eps) or 1)
//   face_values   mdot.mapFaceValues(U.valueAtFace) on boundary faces and
//                 mdot.mapInteriorFaceValues(rhieChowCorrectFace) on interior
//                 faces (SIMPLE.cpp:138-140, operations/rhie_chow.h:47-63,
//                 rhie_chow.cpp:5-25); face flux = value . S_f (vector.h:383-397)
//   correct_*     correctFields (SIMPLE.cpp:218-241)
// All kernels are one thread per face or cell with no atomics.
#include "coupling.h"
#include "devmath.cuh"

namespace pb {

__global__ void d_tensor_kernel(int n, const int* diag_pos, const double* vol, const double* Au, const double* Av,
                                const double* Aw, double* D, int64_t stride) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    int k = diag_pos[c];
    D[c] = vol[c] / (Au[k] + EPSILON);
    D[stride + c] = vol[c] / (Av[k] + EPSILON);
    D[2 * stride + c] = Aw ? vol[c] / (Aw[k] + EPSILON) : 1.0;
}
void launchDTensor(int n, const int* diag_pos, const double* vol, const double* Au, const double* Av,
                   const double* Aw, double* D, int64_t stride, cudaStream_t s) {
    if (n == 0) return;
    d_tensor_kernel<<<ceil_div(n, 256), 256, 0, s>>>(n, diag_pos, vol, Au, Av, Aw, D, stride); countLaunch();
    PB_LAUNCH("d_tensor_kernel");
}

// mdot face values: boundary faces take U.valueAtFace, interior faces the
// Rhie-Chow corrected velocity; empty-patch faces are set to 0.
__global__ void rhie_chow_kernel(const MeshView m, const VectorView U, const TensorView D, const ScalarView P,
                                 double* fd, double* ff) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nf) return;
    D3 u;
    if (f < m.nb) {
        if (m.patch_empty[m.bpatch[f]]) {
            fd[f] = 0.0;
            fd[m.nf + f] = 0.0;
            fd[2 * m.nf + f] = 0.0;
            ff[f] = 0.0;
            return;
        }
        u = vectorFace(m, U, f);
    } else {
        const int o = m.owner[f], n = m.nbr[f];
        D3 Uf = vectorFace(m, U, f);
        D3 gavg = gradFace(m, P, f);
        D3 d_CF = cellCenter(m, n) - cellCenter(m, o);
        double dn = norm(d_CF);
        D3 e = d_CF / dn;
        double gortho = (P.v[n] - P.v[o]) / dn;
        D3 gcalc = gavg + ((gortho - dot(gavg, e)) * e);
        u = Uf - tensorMulFace(m, D, f, gcalc - gavg);
    }
    fd[f] = u.x;
    fd[m.nf + f] = u.y;
    fd[2 * m.nf + f] = u.z;
    ff[f] = dot(u, areaVector(m, f));
}
void launchRhieChow(const MeshView& m, const VectorView& U, const TensorView& D, const ScalarView& P, double* fd,
                    double* ff, cudaStream_t s) {
    if (m.nf == 0) return;
    rhie_chow_kernel<<<ceil_div(m.nf, 256), 256, 0, s>>>(m, U, D, P, fd, ff); countLaunch();
    PB_LAUNCH("rhie_chow_kernel");
}

// U_c -= D_c grad(p')_c
__global__ void correct_u_kernel(int n, ScalarView ux, ScalarView uy, ScalarView uz, const TensorView D,
                                 const ScalarView pp) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    D3 Uc{ux.v[c], uy.v[c], uz.v[c]};
    D3 u = Uc - tensorMulCell(D, c, gradAt(pp, c));
    ux.v[c] = u.x;
    uy.v[c] = u.y;
    uz.v[c] = u.z;
}
// mdot_f -= D_f grad(p')_f on interior faces
__global__ void correct_mdot_kernel(const MeshView m, const TensorView D, const ScalarView pp, double* fd, double* ff) {
    int f = m.nb + blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nf) return;
    D3 v{fd[f], fd[m.nf + f], fd[2 * m.nf + f]};
    D3 u = v - tensorMulFace(m, D, f, gradFace(m, pp, f));
    fd[f] = u.x;
    fd[m.nf + f] = u.y;
    fd[2 * m.nf + f] = u.z;
    ff[f] = dot(u, areaVector(m, f));
}
// p += urf p'
__global__ void correct_p_kernel(int n, double* p, const double* pp, double urf) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n) p[c] = p[c] + (urf * pp[c]);
}
void launchCorrectFields(const MeshView& m, const ScalarView& ux, const ScalarView& uy, const ScalarView& uz,
                         const TensorView& D, const ScalarView& pp, double* fd, double* ff, double* p, double urf,
                         cudaStream_t s) {
    if (m.nc) {
        correct_u_kernel<<<ceil_div(m.nc, 256), 256, 0, s>>>(m.nc, ux, uy, uz, D, pp); countLaunch();
        PB_LAUNCH("correct_u_kernel");
    }
    if (m.nf > m.nb) {
        correct_mdot_kernel<<<ceil_div(m.nf - m.nb, 256), 256, 0, s>>>(m, D, pp, fd, ff); countLaunch();
        PB_LAUNCH("correct_mdot_kernel");
    }
    if (m.nc) {
        correct_p_kernel<<<ceil_div(m.nc, 256), 256, 0, s>>>(m.nc, p, pp.v, urf); countLaunch();
        PB_LAUNCH("correct_p_kernel");
    }
}

}  // namespace pb
