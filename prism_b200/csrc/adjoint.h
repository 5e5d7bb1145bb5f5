// adjoint.h -- discrete adjoint of steady diffusion (transposed assembly and solve).
#pragma once

#include "common.h"
#include "views.h"

namespace pb {

// Quantities of the residual R(phi, kappa, v) = A phi - b of a diffusion
// equation (NonCorrected or Corrected, scalar kappa, least-squares gradient)
// that the adjoint kernels need, all device pointers of one mesh.
struct AdjointParams {
    MeshView m;
    ScalarView phi;        // converged field (values, gradients, face values, BCs)
    ScalarView ks;         // kappa
    const double* pinv;    // least-squares operators: 9 blocks of nc
    const double* w;       // 3 blocks of nk (cell-face entries)
    int64_t nk;
    const int* twin;       // cell-face entry of the same interior face in the other cell, -1 on boundary
    int corrected, corrector;
};

// cf twin map (once per mesh) and transpose positions of the SELL pattern
void buildTwin(const MeshView& m, int* twin, cudaStream_t s);
void buildTransposePositions(int n, int nslices, const int* rowptr, const int* sl_off, const int* sl_col, int* tpos,
                             cudaStream_t s);
// AT[k] = A[tpos[k]] (SELL values of A^T in A's pattern)
void transposeValues(int64_t nnz_padded, const int* tpos, const double* A, double* AT, cudaStream_t s);

// u = pinv^T psi(lambda) (3 blocks of n_pad) and d (n) of the linearised correction terms
void adjointCorrection(const AdjointParams& P, const double* lambda, double* u, double* d, int64_t stride,
                       cudaStream_t s);
// rhs = dJ/dphi - G^T psi - d * lambda   (G: least-squares gradient operator)
void adjointRhs(const AdjointParams& P, const double* dJ, const double* lambda, const double* u, const double* d,
                int64_t stride, double* rhs, cudaStream_t s);
// dJ/dkappa (per cell) and dJ/dv (per boundary face; 0 on empty patches and faces without a value)
void adjointGradients(const AdjointParams& P, const double* lambda, const double* u, int64_t stride, double* gk,
                      double* gv, cudaStream_t s);
// ||a - b||^2 and ||a||^2 into out[0..1] (host), using scratch of >= 2 * 1184 doubles + a counter
void diffNorms(int n, const double* a, const double* b, double* partials, unsigned int* counter, double* dev_out,
               double* host_out, cudaStream_t s);

}  // namespace pb
