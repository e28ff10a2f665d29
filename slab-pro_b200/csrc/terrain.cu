// K0: one-time terrain metric terms in FP64 (compiled with -fmad=false so
// the gradients are the same IEEE operations as the reference).
#include "engine.hpp"

namespace slab {

// Simulation::terrainGradients (src/complex_terrain.cpp:84-100): the gradient
// of cell (i,j) from its four corner nodes, stored at the bottom-left node;
// nodes of the last row and column keep a zero gradient.
// Simulation::terrainTheta (src/complex_terrain.cpp:102-111): theta =
// atan|grad|; the hot loop only ever uses cos(theta), stored directly.
__global__ void k_terrain_metrics(int Nx, int Ny, double one_over_dx, const double* __restrict__ z, double2* __restrict__ grad,
                                  double* __restrict__ cos_t, float4* __restrict__ dem32) {
    const int64_t n = (int64_t)Nx * Ny;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(k / Ny), j = (int)(k % Ny);
        double gx = 0.0, gy = 0.0;
        if (i < Nx - 1 && j < Ny - 1) {
            const double z00 = z[k], z01 = z[k + 1], z10 = z[k + Ny], z11 = z[k + Ny + 1];
            gx = (z10 + z11 - z00 - z01) / 2. * one_over_dx;
            gy = (z01 + z11 - z00 - z10) / 2. * one_over_dx;
        }
        const double c = cos(atan(sqrt(gx * gx + gy * gy)));
        grad[k] = make_double2(gx, gy);
        cos_t[k] = c;
        dem32[k] = make_float4((float)gx, (float)gy, (float)c, (float)z[k]);
    }
}

void compute_terrain_metrics(Terrain& t, cudaStream_t s) {
    const int64_t n = (int64_t)t.Nx * t.Ny;
    int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
    k_terrain_metrics<<<blocks, 256, 0, s>>>(t.Nx, t.Ny, 1. / t.dx, t.z.get(), t.grad.get(), t.cos_t.get(), t.dem32.get());
    SLAB_CUDA(cudaGetLastError());
}

}  // namespace slab
