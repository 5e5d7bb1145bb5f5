// diag.cu -- per-cell diagnostics and cell-to-point interpolation, evaluated
// with the reference's operation order (compiled without FMA contraction).
//
//   div_kernel            ops::div (operations/operations.h:84-100, 144-169)
//   courant_kernel        monitor::courantNumber (monitor/courant.cpp:7-24)
//   cell_to_point_kernel  cellToPoint (export.cpp:73-111)
//
// All three are gathers over a CSR (cell -> faces, vertex -> cells) with one
// thread per output row; they run once per export or monitor call, not per
// solver iteration.
#include "diag.h"
#include "devmath.cuh"

namespace pb {

__global__ void __launch_bounds__(256) div_kernel(const MeshView m, const VectorView U, double* out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    out[c] = fluxSum(m, U, c) / m.vol[c];
}

__global__ void __launch_bounds__(256) courant_kernel(const MeshView m, const VectorView mdot, double dt,
                                                      double* out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    double flux_sum = 0.0;
    for (int q = m.cf_off[c]; q < m.cf_off[c + 1]; ++q) {
        const int f = m.cf_face[q];
        if (f < m.nb && m.patch_empty[m.bpatch[f]]) continue;
        flux_sum += fabs(vectorFlux(m, mdot, f));
    }
    out[c] = 0.5 * dt * flux_sum / m.vol[c];
}

// 1 / max(|x_v - x_c|, eps): recomputed in the second pass instead of stored,
// the same operations give the same weights.
__device__ __forceinline__ double idwWeight(const MeshView& m, D3 xv, int c) {
    return 1.0 / smax(norm(xv - cellCenter(m, c)), EPSILON);
}

template <int NC>
__global__ void __launch_bounds__(256) cell_to_point_kernel(const MeshView m, const PointMapView pm,
                                                            const PointComponents comp, double* out) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= pm.nv) return;
    const D3 xv{pm.vx[v], pm.vy[v], pm.vz[v]};
    const int64_t b = pm.off[v], e = pm.off[v + 1];
    double sum_weights = 0.0;
    for (int64_t i = b; i < e; ++i) sum_weights += idwWeight(m, xv, pm.cell[i]);
    double acc[NC];
#pragma unroll
    for (int k = 0; k < NC; ++k) acc[k] = 0.0;
    for (int64_t i = b; i < e; ++i) {
        const int c = pm.cell[i];
        const double w = idwWeight(m, xv, c) / sum_weights;
#pragma unroll
        for (int k = 0; k < NC; ++k) acc[k] += w * comp.p[k][(int64_t)c * comp.stride];
    }
#pragma unroll
    for (int k = 0; k < NC; ++k) out[v * comp.ncomp + k] = acc[k];
}

void launchDiv(const MeshView& m, const VectorView& U, double* out, cudaStream_t st) {
    if (m.nc == 0) return;
    div_kernel<<<ceil_div(m.nc, 256), 256, 0, st>>>(m, U, out); countLaunch();
    PB_LAUNCH("div_kernel");
}

void launchCourant(const MeshView& m, const VectorView& mdot, double dt, double* out, cudaStream_t st) {
    if (m.nc == 0) return;
    courant_kernel<<<ceil_div(m.nc, 256), 256, 0, st>>>(m, mdot, dt, out); countLaunch();
    PB_LAUNCH("courant_kernel");
}

void launchCellToPoint(const MeshView& m, const PointMapView& pm, const PointComponents& comp, double* out,
                       cudaStream_t st) {
    if (pm.nv == 0 || comp.ncomp == 0) return;
    if (comp.ncomp < 1 || comp.ncomp > MAX_POINT_COMPONENTS) fail(PRISM_BAD_ARG, "n_components must be 1..9");
    const unsigned grid = (unsigned)((pm.nv + 255) / 256);
    if (comp.ncomp == 1 || comp.ncomp == 3 || comp.ncomp == 9) {
        if (comp.ncomp == 1) cell_to_point_kernel<1><<<grid, 256, 0, st>>>(m, pm, comp, out);
        else if (comp.ncomp == 3) cell_to_point_kernel<3><<<grid, 256, 0, st>>>(m, pm, comp, out);
        else cell_to_point_kernel<9><<<grid, 256, 0, st>>>(m, pm, comp, out);
        countLaunch();
    } else {
        // other widths: one component per launch, written at its interleaved slot
        for (int k = 0; k < comp.ncomp; ++k) {
            PointComponents one;
            one.p[0] = comp.p[k];
            one.stride = comp.stride;
            one.ncomp = comp.ncomp;
            cell_to_point_kernel<1><<<grid, 256, 0, st>>>(m, pm, one, out + k);
            countLaunch();
        }
    }
    PB_LAUNCH("cell_to_point_kernel");
}

}  // namespace pb
