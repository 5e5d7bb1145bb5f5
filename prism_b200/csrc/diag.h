// diag.h -- diagnostics of device fields (ops::div, the Courant number) and
// cell-to-point interpolation for export.
#pragma once

#include "views.h"

namespace pb {

// vertex -> adjacent cells (cells in increasing id order) and vertex coordinates
struct PointMapView {
    const double* vx = nullptr;
    const double* vy = nullptr;
    const double* vz = nullptr;
    const int64_t* off = nullptr;  // nv + 1
    const int* cell = nullptr;
    int64_t nv = 0;
};

// Component k of cell c is comp[k][c * stride]; point data is written
// interleaved, out[v * ncomp + k].
constexpr int MAX_POINT_COMPONENTS = 9;
struct PointComponents {
    const double* p[MAX_POINT_COMPONENTS] = {};
    int64_t stride = 1;
    int ncomp = 0;
};

void launchDiv(const MeshView& m, const VectorView& U, double* out, cudaStream_t st);
void launchCourant(const MeshView& m, const VectorView& mdot, double dt, double* out, cudaStream_t st);
void launchCellToPoint(const MeshView& m, const PointMapView& pm, const PointComponents& comp, double* out,
                       cudaStream_t st);

}  // namespace pb
