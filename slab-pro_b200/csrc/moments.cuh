// Particle moments in FP64 on the device: total mass, centre of mass,
// momentum and kinetic energy. These are the conservation and trajectory
// diagnostics of a run (the reference prints only the total volume,
// src/simulation.cpp:473-475); an FP32 run is compared with an FP64 run
// through them frame by frame.
//
// The reduction has a fixed order, so the result is reproducible: each of
// MOM_BLOCKS blocks sums a fixed strided subset of the particles through warp
// shuffles and a fixed-order combine of its warps, then one block adds the
// block partials in index order.
#pragma once

#include "common.cuh"

namespace slab {
namespace {  // each translation unit that reduces moments has its own copy of the kernels

constexpr int MOM_BLOCKS = 296;   // 2 per SM
constexpr int MOM_THREADS = 256;
constexpr int MOM_N = 6;          // m, m x, m y, m vx, m vy, m |v|^2 / 2

// Block-wide sums of MOM_N values in a fixed order; thread 0 gets the result.
__device__ __forceinline__ void mom_block_sum(double (&a)[MOM_N], double (*s)[MOM_THREADS / 32]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < MOM_N; ++q)
        for (int o = 16; o > 0; o >>= 1) a[q] += __shfl_xor_sync(0xffffffffu, a[q], o);
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < MOM_N; ++q) s[q][warp] = a[q];
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < MOM_N; ++q) {
            double t = 0.0;
            for (int w = 0; w < MOM_THREADS / 32; ++w) t += s[q][w];
            a[q] = t;
        }
}

// Stage 1: particle p's position, velocity and mass come from `get`
// (x, y, vx, vy, m as doubles); block b writes its partial to part[b].
template <typename Get> __global__ void __launch_bounds__(MOM_THREADS) k_moments(int Np, Get get, double* part) {
    __shared__ double s[MOM_N][MOM_THREADS / 32];
    double a[MOM_N] = {0, 0, 0, 0, 0, 0};
    for (int p = blockIdx.x * MOM_THREADS + threadIdx.x; p < Np; p += MOM_BLOCKS * MOM_THREADS) {
        double x, y, vx, vy, m;
        get(p, x, y, vx, vy, m);
        a[0] += m;
        a[1] += m * x;
        a[2] += m * y;
        a[3] += m * vx;
        a[4] += m * vy;
        a[5] += 0.5 * m * (vx * vx + vy * vy);
    }
    mom_block_sum(a, s);
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < MOM_N; ++q) part[(size_t)blockIdx.x * MOM_N + q] = a[q];
}

// Stage 2, one block: out = {mass, centre of mass x, y, momentum x, y,
// kinetic energy}.
__global__ void __launch_bounds__(MOM_THREADS) k_moments_final(const double* part, double* out) {
    __shared__ double s[MOM_N][MOM_THREADS / 32];
    double a[MOM_N] = {0, 0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < MOM_BLOCKS; b += MOM_THREADS)
#pragma unroll
        for (int q = 0; q < MOM_N; ++q) a[q] += part[(size_t)b * MOM_N + q];
    mom_block_sum(a, s);
    if (threadIdx.x == 0) {
        const double M = a[0];
        out[0] = M;
        out[1] = M > 0.0 ? a[1] / M : 0.0;
        out[2] = M > 0.0 ? a[2] / M : 0.0;
        out[3] = a[3];
        out[4] = a[4];
        out[5] = a[5];
    }
}

}  // namespace
}  // namespace slab
