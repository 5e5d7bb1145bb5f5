// pattern.h -- device construction of the CSR / SELL-32 matrix pattern.
#pragma once

#include "common.h"

namespace pb {

struct PatternInput {
    int nc, nb, npatch;
    int64_t ncf;           // cell-face entries
    const int* cf_off;     // device, nc+1
    const int* cf_face;    // device
    const int* owner;      // device, nf
    const int* nbr;        // device, nf (-1 on boundary)
    const int* bpatch;     // device, nb
    const int* ppos;       // device, nb: position of the face in its patch's face list
    int nf;                // faces
};

struct PatternOutput {
    int nslices = 0;
    int64_t nnz = 0, sell_nnz = 0;
    DevBuf<int> rowptr, col;       // CSR (column-sorted rows)
    DevBuf<int> sl_off, sl_col;    // SELL-32
    DevBuf<int> diag_pos;          // SELL position of (c, c)
    DevBuf<int> ca_face, ca_pos;   // cell faces in assembly order + SELL positions
    // per face, owner side then neighbour side (-1 where a boundary face has none): the
    // index of the face in that cell's assembly-order list, and the SELL position of the
    // off-diagonal coefficient the face contributes to that cell's row
    DevBuf<int> face_slot, face_pos;
};

void buildPattern(const PatternInput& in, PatternOutput& out, cudaStream_t s);

}  // namespace pb
