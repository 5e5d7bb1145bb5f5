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
// sequential sweep would read. One launch per level, several lanes per cell.
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

// GreenGauss::computeGradAtCell (green_gauss.cpp:47-76) for the cells of one dependency
// level, GG_LPC lanes per cell: each lane evaluates one face's term (phi_b S_f on a
// boundary face of a non-empty patch, S_f^out phi_f with the skewness correction on an
// interior face; nothing on an empty patch) independently of the others, and the cell's
// first lane adds the terms in the cell's face order, so the sum is the sequential
// sweep's, term for term. The face terms' loads are in flight together instead of one
// face after another.
constexpr int GG_LPC = 8;
__global__ void __launch_bounds__(256) gg_level_kernel(const MeshView m, ScalarView s, const int* __restrict__ cells,
                                                       int count) {
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const int idx = gt / GG_LPC, sub = gt % GG_LPC;
    const int lane = threadIdx.x & 31, lead = lane & ~(GG_LPC - 1);
    const bool valid = idx < count;
    const int c = valid ? cells[idx] : 0;
    const int q0 = valid ? m.cf_off[c] : 0;
    const int nq = valid ? m.cf_off[c + 1] - q0 : 0;
    const int nq_max = __reduce_max_sync(0xffffffffu, (unsigned)nq);
    D3 xc{0, 0, 0}, gc{0, 0, 0};
    double phic = 0.0;
    if (valid) {
        xc = cellCenter(m, c);
        phic = s.v[c];
        gc = gradAt(s, c);
    }
    D3 grad{0, 0, 0};
    for (int base = 0; base < nq_max; base += GG_LPC) {
        const int q = base + sub;
        D3 term{0, 0, 0};
        int has = 0;
        if (q < nq) {
            const int f = m.cf_face[q0 + q];
            if (f < m.nb) {
                if (!m.patch_empty[m.bpatch[f]]) {
                    double phi_b = scalarFace(m, s, f);
                    term = phi_b * areaVector(m, f);
                    has = 1;
                }
            } else {
                const int o = m.owner[f];
                const bool own = (o == c);
                const int n = own ? m.nbr[f] : o;
                D3 Sf = areaVector(m, f);
                if (!own) Sf = D3{-Sf.x, -Sf.y, -Sf.z};
                double face_phi = 0.5 * (phic + s.v[n]);
                D3 grad_sum = gc + gradAt(s, n);
                D3 vec = faceCenter(m, f) - (0.5 * (xc + cellCenter(m, n)));
                face_phi += 0.5 * dot(grad_sum, vec);
                term = Sf * face_phi;
                has = 1;
            }
        }
#pragma unroll
        for (int k = 0; k < GG_LPC; ++k) {
            const int src = lead + k;
            const double tx = __shfl_sync(0xffffffffu, term.x, src);
            const double ty = __shfl_sync(0xffffffffu, term.y, src);
            const double tz = __shfl_sync(0xffffffffu, term.z, src);
            const int h = __shfl_sync(0xffffffffu, has, src);
            if (h) grad = grad + D3{tx, ty, tz};
        }
    }
    if (valid && sub == 0) {
        grad = grad / m.vol[c];
        s.g[c] = grad.x;
        s.g[s.gstride + c] = grad.y;
        s.g[2 * s.gstride + c] = grad.z;
    }
}

void launchLeastSquares(const MeshView& m, const ScalarView& s, const double* pinv, const double* w, int64_t nk,
                        cudaStream_t st) {
    if (m.nc == 0) return;
    ls_grad_kernel<<<ceil_div(m.nc, 256), 256, 0, st>>>(m, s, pinv, w, nk); countLaunch();
    PB_LAUNCH("ls_grad_kernel");
}

void launchGreenGauss(const MeshView& m, const ScalarView& s, const int* level_cells,
                      const std::vector<int>& level_off, cudaStream_t st) {
    for (size_t l = 0; l + 1 < level_off.size(); ++l) {
        const int count = level_off[l + 1] - level_off[l];
        if (count == 0) continue;
        gg_level_kernel<<<ceil_div((int64_t)count * GG_LPC, 256), 256, 0, st>>>(m, s, level_cells + level_off[l],
                                                                                count); countLaunch();
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
