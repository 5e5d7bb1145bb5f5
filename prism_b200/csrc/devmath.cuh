// devmath.cuh -- device helpers: 3-vectors, face values of fields and boundary
// handlers, evaluated with the reference's operation order.
#pragma once

#include "common.h"
#include "views.h"

namespace pb {

struct D3 {
    double x, y, z;
};
__device__ __forceinline__ D3 d3(double x, double y, double z) { return {x, y, z}; }
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 operator*(double s, D3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ D3 operator*(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ D3 operator/(D3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ double dot(D3 a, D3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ double norm(D3 a) { return sqrt(dot(a, a)); }
// std::max(a, b) == (a < b) ? b : a -- keeps a NaN first argument (fmax would drop it)
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }

__device__ __forceinline__ D3 cellCenter(const MeshView& m, int c) { return {m.cx[c], m.cy[c], m.cz[c]}; }
__device__ __forceinline__ D3 faceCenter(const MeshView& m, int f) { return {m.fx[f], m.fy[f], m.fz[f]}; }
__device__ __forceinline__ D3 faceNormal(const MeshView& m, int f) { return {m.nx[f], m.ny[f], m.nz[f]}; }
// Face::areaVector (face.h:20): area * normal
__device__ __forceinline__ D3 areaVector(const MeshView& m, int f) {
    double a = m.area[f];
    return {a * m.nx[f], a * m.ny[f], a * m.nz[f]};
}
__device__ __forceinline__ D3 gradAt(const ScalarView& s, int c) {
    return {s.g[c], s.g[s.gstride + c], s.g[2 * s.gstride + c]};
}

// Scalar::valueAtFace (scalar.cpp:189-237) for any face; the boundary handler
// kinds were validated on the host before the launch.
__device__ __forceinline__ double scalarFace(const MeshView& m, const ScalarView& s, int f) {
    if (s.fv) return s.fv[f];
    int o = m.owner[f];
    if (f >= m.nb) {
        double gc = m.gcw[f - m.nb];
        double val = gc * s.v[o];
        val += (1 - gc) * s.v[m.nbr[f]];
        return val;
    }
    int p = m.bpatch[f];
    int k = s.bc_kind[p];
    if (k == PRISM_BC_FIXED || k == PRISM_BC_NOSLIP) return s.bc_val[p];
    return s.v[o];  // symmetry / outlet / zero-gradient: owner value
}

// GeneralVector::valueAtFace (vector.h:188-226, vector_boundary.h:75-115)
__device__ __forceinline__ D3 vectorFace(const MeshView& m, const VectorView& U, int f) {
    if (U.fd) return {U.fd[f], U.fd[m.nf + f], U.fd[2 * m.nf + f]};
    if (f < m.nb) {
        int p = m.bpatch[f];
        int k = U.bc_kind[p];
        if (k == PRISM_BC_FIXED || k == PRISM_BC_NOSLIP) return {U.bc_vec[3 * p], U.bc_vec[3 * p + 1], U.bc_vec[3 * p + 2]};
        int o = m.owner[f];
        D3 Uc{U.c[0].v[o], U.c[1].v[o], U.c[2].v[o]};
        if (k == PRISM_BC_SYMMETRY) {
            D3 n = faceNormal(m, f);
            return Uc - dot(Uc, n) * n;
        }
        return Uc;
    }
    return {scalarFace(m, U.c[0], f), scalarFace(m, U.c[1], f), scalarFace(m, U.c[2], f)};
}

// GeneralVector::fluxAtFace (vector.h:238-290)
__device__ __forceinline__ double vectorFlux(const MeshView& m, const VectorView& U, int f) {
    if (U.ff) return U.ff[f];
    if (f < m.nb) {
        int k = U.bc_kind[m.bpatch[f]];
        if (k == PRISM_BC_NOSLIP || k == PRISM_BC_SYMMETRY) return 0.0;
    }
    return dot(vectorFace(m, U, f), areaVector(m, f));
}

// ops::div flux sum (operations.h:144-169): signed fluxAtFace over the cell's
// non-empty faces, in the cell's face order
__device__ __forceinline__ double fluxSum(const MeshView& m, const VectorView& U, int c) {
    double sum = 0.0;
    for (int q = m.cf_off[c]; q < m.cf_off[c + 1]; ++q) {
        int f = m.cf_face[q];
        if (f < m.nb && m.patch_empty[m.bpatch[f]]) continue;
        double flux = vectorFlux(m, U, f);
        if (m.owner[f] != c) flux = -flux;
        sum += flux;
    }
    return sum;
}

// T^T v with a cell or an interpolated face tensor (diffusion_coeff.cpp:21-30).
__device__ __forceinline__ double tget(const TensorView& T, int i, int j, int c) {
    if (T.diag) return i == j ? T.d[i * T.stride + c] : 0.0;
    return T.d[(3 * i + j) * T.stride + c];
}
__device__ __forceinline__ D3 tensorTmulCell(const TensorView& T, int c, D3 v) {
    D3 r;
    r.x = (tget(T, 0, 0, c) * v.x + tget(T, 1, 0, c) * v.y) + tget(T, 2, 0, c) * v.z;
    r.y = (tget(T, 0, 1, c) * v.x + tget(T, 1, 1, c) * v.y) + tget(T, 2, 1, c) * v.z;
    r.z = (tget(T, 0, 2, c) * v.x + tget(T, 1, 2, c) * v.y) + tget(T, 2, 2, c) * v.z;
    return r;
}
// Tensor::valueAtFace (tensor.cpp:58-77): gc*T_O + (1-gc)*T_N on interior faces
__device__ __forceinline__ double tfaceget(const MeshView& m, const TensorView& T, int i, int j, int f) {
    int o = m.owner[f];
    if (f < m.nb) return tget(T, i, j, o);
    double gc = m.gcw[f - m.nb];
    return (gc * tget(T, i, j, o)) + ((1 - gc) * tget(T, i, j, m.nbr[f]));
}
__device__ __forceinline__ D3 tensorTmulFace(const MeshView& m, const TensorView& T, int f, D3 v) {
    D3 r;
    r.x = (tfaceget(m, T, 0, 0, f) * v.x + tfaceget(m, T, 1, 0, f) * v.y) + tfaceget(m, T, 2, 0, f) * v.z;
    r.y = (tfaceget(m, T, 0, 1, f) * v.x + tfaceget(m, T, 1, 1, f) * v.y) + tfaceget(m, T, 2, 1, f) * v.z;
    r.z = (tfaceget(m, T, 0, 2, f) * v.x + tfaceget(m, T, 1, 2, f) * v.y) + tfaceget(m, T, 2, 2, f) * v.z;
    return r;
}
// T v (not transposed), cell and face
__device__ __forceinline__ D3 tensorMulCell(const TensorView& T, int c, D3 v) {
    D3 r;
    r.x = (tget(T, 0, 0, c) * v.x + tget(T, 0, 1, c) * v.y) + tget(T, 0, 2, c) * v.z;
    r.y = (tget(T, 1, 0, c) * v.x + tget(T, 1, 1, c) * v.y) + tget(T, 1, 2, c) * v.z;
    r.z = (tget(T, 2, 0, c) * v.x + tget(T, 2, 1, c) * v.y) + tget(T, 2, 2, c) * v.z;
    return r;
}
__device__ __forceinline__ D3 tensorMulFace(const MeshView& m, const TensorView& T, int f, D3 v) {
    D3 r;
    r.x = (tfaceget(m, T, 0, 0, f) * v.x + tfaceget(m, T, 0, 1, f) * v.y) + tfaceget(m, T, 0, 2, f) * v.z;
    r.y = (tfaceget(m, T, 1, 0, f) * v.x + tfaceget(m, T, 1, 1, f) * v.y) + tfaceget(m, T, 1, 2, f) * v.z;
    r.z = (tfaceget(m, T, 2, 0, f) * v.x + tfaceget(m, T, 2, 1, f) * v.y) + tfaceget(m, T, 2, 2, f) * v.z;
    return r;
}

// IGradient::gradAtFace (gradient.cpp:15-51 + gradient/boundary.cpp:6-34)
__device__ __forceinline__ D3 gradFace(const MeshView& m, const ScalarView& s, int f) {
    int o = m.owner[f];
    if (f >= m.nb) {
        double gc = m.gcw[f - m.nb];
        return (gc * gradAt(s, o)) + ((1. - gc) * gradAt(s, m.nbr[f]));
    }
    int k = s.bc_kind[m.bpatch[f]];
    D3 grad_c = gradAt(s, o);
    if (k == PRISM_BC_FIXED || k == PRISM_BC_NOSLIP) {
        D3 d_Cf = faceCenter(m, f) - cellCenter(m, o);
        D3 e = d_Cf / norm(d_Cf);
        double phi_b = scalarFace(m, s, f);
        double phi_C = s.v[o];
        return (grad_c - dot(grad_c, e) * e) + ((phi_b - phi_C) / norm(d_Cf)) * e;
    }
    return grad_c;
}

}  // namespace pb
