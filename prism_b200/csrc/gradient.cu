// gradient.cu -- cell gradients as deterministic cell-owned gathers.
//
// Least squares (gradient/least_squares.cpp:63-100): grad_c = pinv_c * sum_e
// w_e (phi_e - phi_c) over the cell's interior faces and non-empty boundary
// faces, in the cell's face order; pinv and w are built once per mesh on the
// host (least_squares.cpp:12-61).
//
// Green-Gauss with skewness correction (gradient/green_gauss.cpp:11-88) is an
// in-place sweep in cell order: cell c reads the already-updated gradient of
// every lower-numbered neighbour and the previous gradient of every higher one.
// The sweep is run level by level over the lower-neighbour dependency DAG
// (level[c] = 1 + max level of its lower-numbered neighbours): cells of one level
// never neighbour each other, so each cell reads exactly the values the
// sequential sweep would read. Few levels: one launch per level; many (the
// hyperplanes of a structured 3-D mesh: 382 at 128^3): one cooperative launch
// with a grid barrier between levels.
#include <cooperative_groups.h>

#include <cstdlib>

#include "devmath.cuh"
#include "gradient.h"

namespace pb {

__global__ void __launch_bounds__(256) ls_grad_kernel(const MeshView m, ScalarView s, const double* __restrict__ pinv,
                                                      const double* __restrict__ w, int64_t nk) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const double phic = s.v[c];
    D3 b{0, 0, 0};
    for (int q = m.cf_off[c]; q < m.cf_off[c + 1]; ++q) {
        int f = m.cf_face[q];
        double other;
        if (f >= m.nb) {
            int o = m.owner[f];
            other = s.v[o == c ? m.nbr[f] : o];
        } else {
            if (m.patch_empty[m.bpatch[f]]) continue;
            other = scalarFace(m, s, f);
        }
        D3 wq{w[q], w[nk + q], w[2 * nk + q]};
        b = b + wq * (other - phic);
    }
    int64_t n = m.nc;
    for (int i = 0; i < 3; ++i) {
        double gi = (pinv[(3 * i) * n + c] * b.x + pinv[(3 * i + 1) * n + c] * b.y) + pinv[(3 * i + 2) * n + c] * b.z;
        s.g[i * s.gstride + c] = gi;
    }
}

// gradient at a cell, read through L2 (values written by other blocks of the same launch)
__device__ __forceinline__ D3 gradAtL2(const ScalarView& s, int c) {
    return D3{__ldcg(s.g + c), __ldcg(s.g + s.gstride + c), __ldcg(s.g + 2 * s.gstride + c)};
}

// GreenGauss::computeGradAtCell (green_gauss.cpp:47-76) for cell c; L2: read the gradients
// through L2 (the sweep kernel, where other blocks wrote them in this launch)
template <bool L2>
__device__ __forceinline__ void ggCell(const MeshView& m, const ScalarView& s, int c) {
    const D3 xc = cellCenter(m, c);
    const double phic = s.v[c];
    const D3 gc = L2 ? gradAtL2(s, c) : gradAt(s, c);
    D3 grad{0, 0, 0};
    for (int q = m.cf_off[c]; q < m.cf_off[c + 1]; ++q) {
        int f = m.cf_face[q];
        if (f < m.nb) {
            if (m.patch_empty[m.bpatch[f]]) continue;
            double phi_b = scalarFace(m, s, f);
            grad = grad + phi_b * areaVector(m, f);
            continue;
        }
        int o = m.owner[f];
        bool own = (o == c);
        int n = own ? m.nbr[f] : o;
        D3 Sf = areaVector(m, f);
        if (!own) Sf = D3{-Sf.x, -Sf.y, -Sf.z};
        double face_phi = 0.5 * (phic + s.v[n]);
        D3 grad_sum = gc + (L2 ? gradAtL2(s, n) : gradAt(s, n));
        D3 vec = faceCenter(m, f) - (0.5 * (xc + cellCenter(m, n)));
        face_phi += 0.5 * dot(grad_sum, vec);
        grad = grad + Sf * face_phi;
    }
    grad = grad / m.vol[c];
    s.g[c] = grad.x;
    s.g[s.gstride + c] = grad.y;
    s.g[2 * s.gstride + c] = grad.z;
}

__global__ void __launch_bounds__(256) gg_level_kernel(const MeshView m, ScalarView s, const int* __restrict__ cells,
                                                       int count) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    ggCell<false>(m, s, cells[t]);
}

// The whole sweep in one cooperative launch: the levels in order, separated by grid
// barriers (every block is co-resident and takes every barrier), so level l reads the
// gradients level l - 1 wrote exactly as the one-launch-per-level sweep does.
__global__ void __launch_bounds__(256) gg_sweep_kernel(const MeshView m, ScalarView s, const int* __restrict__ cells,
                                                       const int* __restrict__ level_off, int nlevels) {
    namespace cg = cooperative_groups;
    const int nthreads = (int)(gridDim.x * blockDim.x);
    const int t0 = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    for (int l = 0; l < nlevels; ++l) {
        const int end = level_off[l + 1];
        for (int t = level_off[l] + t0; t < end; t += nthreads) ggCell<true>(m, s, cells[t]);
        if (l + 1 < nlevels) cg::this_grid().sync();
    }
}

void launchLeastSquares(const MeshView& m, const ScalarView& s, const double* pinv, const double* w, int64_t nk,
                        cudaStream_t st) {
    if (m.nc == 0) return;
    ls_grad_kernel<<<ceil_div(m.nc, 256), 256, 0, st>>>(m, s, pinv, w, nk); countLaunch();
    PB_LAUNCH("ls_grad_kernel");
}

// sweeps of more levels than this run as one cooperative launch (PRISM_GG_COOP_LEVELS; 0, the
// default: never -- on the 128^3 mesh the grid barriers cost more than the launches they replace)
int ggCoopLevels() {
    static const int v = [] {
        const char* e = std::getenv("PRISM_GG_COOP_LEVELS");
        return e && e[0] ? std::max(0, std::atoi(e)) : 0;
    }();
    return v;
}

void launchGreenGauss(const MeshView& m, const ScalarView& s, const int* level_cells,
                      const std::vector<int>& level_off, const int* level_off_dev, cudaStream_t st) {
    const int nlevels = (int)level_off.size() - 1;
    if (nlevels <= 0) return;
    if (ggCoopLevels() > 0 && nlevels > ggCoopLevels() && level_off_dev) {
        static const int blocks = [] {
            int dev = 0, sms = 148, per = 1;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, gg_sweep_kernel, 256, 0) != cudaSuccess || per < 1)
                per = 1;
            cudaGetLastError();
            return per * sms;
        }();
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3((unsigned)blocks);
        cfg.blockDim = dim3(256);
        cfg.stream = st;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeCooperative;
        at[0].val.cooperative = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        PB_CUDA(cudaLaunchKernelEx(&cfg, gg_sweep_kernel, m, s, level_cells, level_off_dev, nlevels));
        countLaunch();
        PB_LAUNCH("gg_sweep_kernel");
        return;
    }
    for (int l = 0; l < nlevels; ++l) {
        int count = level_off[l + 1] - level_off[l];
        if (count == 0) continue;
        gg_level_kernel<<<ceil_div(count, 256), 256, 0, st>>>(m, s, level_cells + level_off[l], count); countLaunch();
    }
    PB_LAUNCH("gg_level_kernel");
}

// valueAtFace / fluxAtFace for every face (empty-patch faces give 0)
__global__ void scalar_faces_kernel(const MeshView m, ScalarView s, double* out) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nf) return;
    out[f] = (f < m.nb && m.patch_empty[m.bpatch[f]]) ? 0.0 : scalarFace(m, s, f);
}
__global__ void vector_flux_kernel(const MeshView m, VectorView U, double* out) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nf) return;
    out[f] = (f < m.nb && m.patch_empty[m.bpatch[f]]) ? 0.0 : vectorFlux(m, U, f);
}
void launchScalarFaces(const MeshView& m, const ScalarView& s, double* out, cudaStream_t st) {
    if (m.nf == 0) return;
    scalar_faces_kernel<<<ceil_div(m.nf, 256), 256, 0, st>>>(m, s, out); countLaunch();
    PB_LAUNCH("scalar_faces_kernel");
}
void launchVectorFlux(const MeshView& m, const VectorView& U, double* out, cudaStream_t st) {
    if (m.nf == 0) return;
    vector_flux_kernel<<<ceil_div(m.nf, 256), 256, 0, st>>>(m, U, out); countLaunch();
    PB_LAUNCH("vector_flux_kernel");
}

}  // namespace pb
