// gradient.h -- launch interface of the gradient and face-value kernels.
#pragma once

#include <vector>

#include "common.h"
#include "views.h"

namespace pb {

void launchLeastSquares(const MeshView& m, const ScalarView& s, const double* pinv, const double* w, int64_t nk,
                        cudaStream_t st);
void launchGreenGauss(const MeshView& m, const ScalarView& s, const int* level_cells,
                      const std::vector<int>& level_off, cudaStream_t st);
void launchScalarFaces(const MeshView& m, const ScalarView& s, double* out, cudaStream_t st);
void launchVectorFlux(const MeshView& m, const VectorView& U, double* out, cudaStream_t st);

}  // namespace pb
