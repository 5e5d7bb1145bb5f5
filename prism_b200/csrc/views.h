// views.h -- plain-pointer views of device data passed to kernels by value.
//
// HBM layout (all structure-of-arrays, one array per component):
//   faces  [0, nne) non-empty boundary | [nne, nb) empty boundary | [nb, nf) interior
//          owner, nbr (-1 on boundary), bpatch (boundary faces), area, normal xyz,
//          centre xyz; gcw = geometric weight of interior faces (index f - nb)
//   cells  centre xyz, volume; cell->face lists (reference local order) with, per
//          entry, the SELL position of the (cell, neighbour) coefficient
//   matrix SELL-32: slice s holds rows [32s, 32s+32); entry j of row r sits at
//          sl_off[s] + 32*j + (r & 31); rows are column-sorted (CSR order), padded
//          with (col = row, value 0) up to the slice width.
#pragma once

#include <cstdint>

namespace pb {

struct MeshView {
    int nc, nf, nb, nne, npatch, nslices;
    const int* owner;
    const int* nbr;
    const int* bpatch;
    const unsigned char* patch_empty;
    const double* area;
    const double* nx;
    const double* ny;
    const double* nz;
    const double* fx;
    const double* fy;
    const double* fz;
    const double* cx;
    const double* cy;
    const double* cz;
    const double* vol;
    const double* gcw;
    const int* cf_off;
    const int* cf_face;
    const int* cf_pos;   // SELL position of (c, other) for interior entries, -1 on boundary
    const int* diag_pos; // SELL position of (c, c)
    const int* sl_off;   // nslices + 1
    const int* sl_col;
};

// field::Scalar
struct ScalarView {
    double* v;             // cell values
    const double* fv;      // face values or nullptr (setFaceValues)
    double* g;             // cell gradients, 3 blocks of stride gstride
    int64_t gstride;
    const int* bc_kind;    // per patch, PRISM_BC_*
    const double* bc_val;  // per patch, resolved scalar value (component of a vector BC)
    const double* bc_vec;  // per patch, 3 values (fixed-gradient wall gradient)
};

// field::Vector: components + optional face values / face fluxes
struct VectorView {
    ScalarView c[3];
    const double* fd;      // 3 blocks of nf, or nullptr
    const double* ff;      // nf, or nullptr
    const int* bc_kind;
    const double* bc_vec;  // per patch, 3 values
};

// field::Tensor (9 blocks of stride n, or 3 diagonal blocks when diag != 0)
struct TensorView {
    const double* d;
    int64_t stride;
    int diag;
};

}  // namespace pb
