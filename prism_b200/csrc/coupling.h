// coupling.h -- launch interface of the pressure-velocity coupling kernels.
#pragma once

#include "common.h"
#include "views.h"

namespace pb {

void launchDTensor(int n, const int* diag_pos, const double* vol, const double* Au, const double* Av,
                   const double* Aw, double* D, int64_t stride, cudaStream_t s);
void launchRhieChow(const MeshView& m, const VectorView& U, const TensorView& D, const ScalarView& P, double* fd,
                    double* ff, cudaStream_t s);
void launchCorrectFields(const MeshView& m, const ScalarView& ux, const ScalarView& uy, const ScalarView& uz,
                         const TensorView& D, const ScalarView& pp, double* fd, double* ff, double* p, double urf,
                         cudaStream_t s);

}  // namespace pb
