// reduce.cuh -- deterministic grid-wide reductions shared by the solver kernels.
//
// A reducing kernel accumulates per-thread partial sums (or maxima) of NV
// values, then calls reduceLast(): every block reduces its threads in a fixed
// order and publishes one partial per value, and the last block to arrive
// (an atomic ticket) reduces the block partials in block order. The result is
// bitwise the same on every run for a given grid, with no floating-point
// atomics. The caller's scalar epilogue runs in thread 0 of the last block.
#pragma once

#include "common.h"

namespace pb {

__device__ __forceinline__ double warpSum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warpMax(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// Block-reduce NV sums (or maxima), publish the block partial, and let the last
// block to arrive reduce all partials in block order. Returns true in the last
// block, where out[] holds the grid totals in every thread. partials holds
// gridDim.x * NV doubles; counter starts at 0 and is left at 0.
template <int NV, bool MAX, int BLOCK = 256>
__device__ bool reduceLast(double (&v)[NV], double* partials, unsigned int* counter, double (&out)[NV]) {
    constexpr int NW = BLOCK / 32;
    __shared__ double sh[NV][NW];
    __shared__ int is_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < NV; ++k) {
        double x = MAX ? warpMax(v[k]) : warpSum(v[k]);
        if (lane == 0) sh[k][warp] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < NV; ++k) {
            double s = sh[k][0];
            for (int w = 1; w < NW; ++w) s = MAX ? fmax(s, sh[k][w]) : s + sh[k][w];
            partials[blockIdx.x * NV + k] = s;
        }
        __threadfence();
        unsigned int t = atomicAdd(counter, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    double acc[NV];
    for (int k = 0; k < NV; ++k) {
        acc[k] = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += BLOCK) {
            double x = __ldcg(&partials[b * NV + k]);
            acc[k] = MAX ? fmax(acc[k], x) : acc[k] + x;
        }
    }
    __syncthreads();
    for (int k = 0; k < NV; ++k) {
        double x = MAX ? warpMax(acc[k]) : warpSum(acc[k]);
        if (lane == 0) sh[k][warp] = x;
    }
    __syncthreads();
    for (int k = 0; k < NV; ++k) {
        double s = sh[k][0];
        for (int w = 1; w < NW; ++w) s = MAX ? fmax(s, sh[k][w]) : s + sh[k][w];
        out[k] = s;
    }
    if (threadIdx.x == 0) *counter = 0u;
    return true;
}

}  // namespace pb
