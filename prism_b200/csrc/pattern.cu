// pattern.cu -- the matrix sparsity pattern, built on the device.
//
// The reference builds its matrix with LinearSystem::insert + setFromTriplets
// (linear.cpp:17-28) on every assembly; the pattern that results is, per row,
// the diagonal plus the face neighbours, sorted by column. Here it is built
// once per mesh:
//   1. row_kernel: each cell gathers {c} U neighbours from its face list,
//      sorts and de-duplicates them -> row length;
//   2. exclusive scans (CUB) give the CSR row pointer and, from the per-slice
//      maximum row length, the SELL-32 slice offsets;
//   3. fill_kernel writes CSR columns, SELL columns (padding: col = row,
//      value 0), the SELL position of the diagonal and of every (cell,
//      neighbour) coefficient, and the cell's faces in assembly order
//      (boundary faces by (patch, position in patch), then interior by id).
#include <cub/cub.cuh>

#include "pattern.h"

namespace pb {

namespace {

constexpr int MAXF = 32;  // faces per cell handled by the pattern kernels

__device__ int sortedRow(int c, const int* cf_off, const int* cf_face, const int* owner, const int* nbr, int nb,
                         int* cols) {
    int n = 0;
    cols[n++] = c;
    for (int q = cf_off[c]; q < cf_off[c + 1]; ++q) {
        int f = cf_face[q];
        if (f < nb) continue;
        int o = owner[f];
        cols[n++] = (o == c) ? nbr[f] : o;
    }
    for (int i = 1; i < n; ++i) {  // insertion sort
        int v = cols[i], j = i - 1;
        while (j >= 0 && cols[j] > v) {
            cols[j + 1] = cols[j];
            --j;
        }
        cols[j + 1] = v;
    }
    int u = 1;
    for (int i = 1; i < n; ++i)
        if (cols[i] != cols[u - 1]) cols[u++] = cols[i];
    return u;
}

__global__ void row_kernel(int nc, const int* cf_off, const int* cf_face, const int* owner, const int* nbr, int nb,
                           int* rowlen, int* bad) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    if (cf_off[c + 1] - cf_off[c] >= MAXF) {
        atomicExch(bad, 1);
        rowlen[c] = 1;
        return;
    }
    int cols[MAXF];
    rowlen[c] = sortedRow(c, cf_off, cf_face, owner, nbr, nb, cols);
}

__global__ void slice_kernel(int nc, int nslices, const int* rowlen, int* slice_entries) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslices) return;
    int w = 0;
    for (int l = 0; l < 32; ++l) {
        int r = s * 32 + l;
        if (r < nc) w = max(w, rowlen[r]);
    }
    slice_entries[s] = 32 * w;
}

__global__ void fill_kernel(int nc, int nslices, const int* cf_off, const int* cf_face, const int* owner,
                            const int* nbr, int nb, int npatch, const int* bpatch, const int* ppos,
                            const int* rowptr, const int* sl_off, int* csr_col, int* sl_col, int* diag_pos,
                            int* ca_face, int* ca_pos) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nslices * 32) return;
    const int s = r >> 5, lane = r & 31;
    const int base = sl_off[s], width = (sl_off[s + 1] - base) >> 5;
    if (r >= nc) {
        for (int j = 0; j < width; ++j) sl_col[base + 32 * j + lane] = 0;
        return;
    }
    int cols[MAXF];
    int len = sortedRow(r, cf_off, cf_face, owner, nbr, nb, cols);
    for (int j = 0; j < len; ++j) {
        csr_col[rowptr[r] + j] = cols[j];
        sl_col[base + 32 * j + lane] = cols[j];
        if (cols[j] == r) diag_pos[r] = base + 32 * j + lane;
    }
    for (int j = len; j < width; ++j) sl_col[base + 32 * j + lane] = r;
    // faces in assembly order
    const int q0 = cf_off[r], nq = cf_off[r + 1] - q0;
    long long keys[MAXF];
    int fs[MAXF];
    for (int i = 0; i < nq; ++i) {
        int f = cf_face[q0 + i];
        fs[i] = f;
        keys[i] = f < nb ? ((long long)bpatch[f] << 32) | (unsigned)ppos[f] : ((long long)npatch << 32) | (unsigned)f;
    }
    for (int i = 1; i < nq; ++i) {
        long long k = keys[i];
        int f = fs[i], j = i - 1;
        while (j >= 0 && keys[j] > k) {
            keys[j + 1] = keys[j];
            fs[j + 1] = fs[j];
            --j;
        }
        keys[j + 1] = k;
        fs[j + 1] = f;
    }
    for (int i = 0; i < nq; ++i) {
        int f = fs[i];
        ca_face[q0 + i] = f;
        int pos = -1;
        if (f >= nb) {
            int o = owner[f];
            int other = (o == r) ? nbr[f] : o;
            for (int j = 0; j < len; ++j)
                if (cols[j] == other) pos = base + 32 * j + lane;
        }
        ca_pos[q0 + i] = pos;
    }
}

// face -> (cell, face) entries of the assembly-order lists, both sides
__global__ void face_slots_kernel(int nc, const int* cf_off, const int* ca_face, const int* ca_pos, const int* owner,
                                  int* face_slot, int* face_pos) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    for (int q = cf_off[c]; q < cf_off[c + 1]; ++q) {
        const int f = ca_face[q];
        const int side = owner[f] == c ? 0 : 1;
        face_slot[2 * f + side] = q;
        face_pos[2 * f + side] = ca_pos[q];
    }
}

}  // namespace

void buildPattern(const PatternInput& in, PatternOutput& out, cudaStream_t s) {
    const int nc = in.nc;
    const int nslices = ceil_div(nc, 32);
    DevBuf<int> rowlen(nc + 1), bad(1), slice_entries(nslices + 1);
    PB_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
    PB_CUDA(cudaMemsetAsync(rowlen.p + nc, 0, sizeof(int), s));
    PB_CUDA(cudaMemsetAsync(slice_entries.p + nslices, 0, sizeof(int), s));
    row_kernel<<<ceil_div(nc, 256), 256, 0, s>>>(nc, in.cf_off, in.cf_face, in.owner, in.nbr, in.nb, rowlen.p, bad.p); countLaunch();
    slice_kernel<<<ceil_div(nslices, 256), 256, 0, s>>>(nc, nslices, rowlen.p, slice_entries.p); countLaunch();
    PB_LAUNCH("pattern row/slice kernels");
    out.rowptr.alloc(nc + 1);
    out.sl_off.alloc(nslices + 1);
    size_t tmp_bytes = 0, t2 = 0;
    PB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, rowlen.p, out.rowptr.p, nc + 1, s));
    PB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, t2, slice_entries.p, out.sl_off.p, nslices + 1, s));
    DevBuf<unsigned char> tmp(std::max(tmp_bytes, t2));
    PB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tmp_bytes, rowlen.p, out.rowptr.p, nc + 1, s));
    PB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, t2, slice_entries.p, out.sl_off.p, nslices + 1, s));
    int h[2];
    PB_CUDA(cudaMemcpyAsync(&h[0], out.rowptr.p + nc, sizeof(int), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaMemcpyAsync(&h[1], out.sl_off.p + nslices, sizeof(int), cudaMemcpyDeviceToHost, s));
    int hbad = 0;
    PB_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
    if (hbad) fail(PRISM_INVALID_MESH, "a cell has more faces than the pattern builder supports");
    out.nnz = h[0];
    out.sell_nnz = h[1];
    out.nslices = nslices;
    out.col.alloc(out.nnz);
    out.sl_col.alloc(out.sell_nnz);
    out.diag_pos.alloc(nc);
    out.ca_face.alloc(in.ncf);
    out.ca_pos.alloc(in.ncf);
    fill_kernel<<<ceil_div((int64_t)nslices * 32, 256), 256, 0, s>>>(
        nc, nslices, in.cf_off, in.cf_face, in.owner, in.nbr, in.nb, in.npatch, in.bpatch, in.ppos, out.rowptr.p,
        out.sl_off.p, out.col.p, out.sl_col.p, out.diag_pos.p, out.ca_face.p, out.ca_pos.p); countLaunch();
    PB_LAUNCH("pattern fill_kernel");
    out.face_slot.alloc(2 * (size_t)std::max(in.nf, 1));
    out.face_pos.alloc(2 * (size_t)std::max(in.nf, 1));
    PB_CUDA(cudaMemsetAsync(out.face_slot.p, 0xff, 2 * (size_t)std::max(in.nf, 1) * sizeof(int), s));
    PB_CUDA(cudaMemsetAsync(out.face_pos.p, 0xff, 2 * (size_t)std::max(in.nf, 1) * sizeof(int), s));
    face_slots_kernel<<<ceil_div(nc, 256), 256, 0, s>>>(nc, in.cf_off, out.ca_face.p, out.ca_pos.p, in.owner,
                                                        out.face_slot.p, out.face_pos.p); countLaunch();
    PB_LAUNCH("pattern face_slots_kernel");
    PB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace pb
