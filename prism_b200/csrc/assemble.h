// assemble.h -- launch interface of the assembly kernels.
#pragma once

#include "common.h"
#include "views.h"

namespace pb {

constexpr int MAX_SOURCES = 4;

struct ConvDesc {
    int scheme;
    VectorView U;
};
struct DiffDesc {
    int corrected, corrector, kappa_tensor;
    ScalarView ks;
    TensorView kt;
};
struct SourceDesc {
    int kind, sign, coord;
    ScalarView s;
    VectorView U;
};
// temporal::BackwardEuler / AdamMoulton: previous time steps of the field
struct TemporalDesc {
    int second_order;      // AdamMoulton with two history steps
    double dt;
    const double* prev;    // step 0 of the history
    const double* prev2;   // step 1 (second order only)
};
enum { SCH_CONV = 0, SCH_DIFF = 1, SCH_TEMPORAL = 2 };

struct AssembleParams {
    MeshView m;
    ScalarView phi;
    int phi_coord;
    int has_conv, has_diff, conv_first, need_grad;
    int has_temporal;
    int nsch, order[3];  // schemes in registration order (SCH_*): Transport::updateCoeffs sums in this order
    TemporalDesc tm;
    int nsrc, symmetry, accumulate;
    ConvDesc conv;
    DiffDesc diff;
    SourceDesc src[MAX_SOURCES];
    const int* ca_off;  // cell -> faces in insertion order
    const int* ca_face;
    const int* ca_pos;  // SELL position of (c, other), -1 on boundary
    const int* face_slot;  // per face, owner / neighbour side: index of the face in that cell's list
    const int* face_pos;   // per face, owner / neighbour side: SELL position of the off-diagonal
    double* rec;        // 4 doubles per list entry: the face's terms of that row (zero on empty faces)
    double* A;          // SELL values
    double* b;
    double* bconv;      // accumulated scheme right-hand sides
    double* bdiff;
};

void launchAssemble(const AssembleParams& P, cudaStream_t s);
void launchRelax(double* A, double* b, const int* diag_pos, const double* phi, double alpha, int n, cudaStream_t s);
void launchPin(double* A, double* b, int pos, int row, double ref_value, cudaStream_t s);
void launchPinDev(double* A, double* b, const int* diag_pos, int row, double ref_value, cudaStream_t s);

}  // namespace pb
