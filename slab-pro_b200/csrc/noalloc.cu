// slab_initial_grid_static: the t=0 grid of the FP32 split path (P2G in
// fixed point + the grid update with dt = 0) computed without allocating any
// memory. Inputs and outputs are the caller's device buffers; the only
// scratch -- the fixed-point node sums, per-cell counts and the scale
// bounds -- lives in one file-scope __device__ array of fixed size.
//
// Who needs this: programs that embed the engine into a host framework that
// owns the GPU heap (it reserves all device memory up front and forbids any
// further cudaMalloc / cudaFree from libraries), and real-time or certified
// control loops that may not allocate after start-up. They can still get the
// frame-0 grid of a particle set from buffers they already own.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

#include "common.cuh"
#include "slab_gpu.h"

namespace slab {

void set_thread_error(const std::string& msg);  // capi.cu: message for slab_last_error(NULL)

namespace {

constexpr int SQ = 7;                         // sums per node: m, m vx, m vy, m h, Fx, Fy, m vz
constexpr int HDR = 16;                       // header ints: 7 bounds, max cell count, error flag
constexpr int MAXN = SLAB_STATIC_MAX_NODES;   // nodes of the largest box
// [0, HDR) header | [HDR, HDR+MAXN) particle count per cell | then hi sums
// (SQ planes) and lo sums (SQ planes) of MAXN nodes each.
constexpr size_t SCRATCH_INTS = HDR + (size_t)MAXN * (1 + 2 * SQ);

// Shared by every call in this process on this device: each call clears the
// part it uses first, and calls that overlap on the GPU race on it.
static __device__ __align__(256) int g_scratch[SCRATCH_INTS];

struct Box {
    int i0, j0, nI, nJ;
};

__global__ void k_clear(int* s, int nodes) {
    const int64_t n = HDR + (int64_t)nodes * (1 + 2 * SQ);
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        // node planes are laid out for MAXN nodes; clear only the used prefix of each
        int64_t idx;
        if (k < HDR + nodes) {
            idx = k;
        } else {
            const int64_t r = k - HDR - nodes;
            idx = HDR + MAXN + (r / nodes) * MAXN + (r % nodes);
        }
        s[idx] = 0;
    }
}

// terrain slope terms of the cell (i, j) from the FP64 DEM
// (src/complex_terrain.cpp:84-111): cell gradient from its corners, cos of
// the slope angle
__device__ __forceinline__ void cell_slope(const double* z, int Nx, int Ny, double ood, int i, int j, float& gx, float& gy, float& ct) {
    double dgx = 0.0, dgy = 0.0;
    if (i < Nx - 1 && j < Ny - 1) {
        const int64_t k = (int64_t)i * Ny + j;
        const double z00 = z[k], z01 = z[k + 1], z10 = z[k + Ny], z11 = z[k + Ny + 1];
        dgx = (z10 + z11 - z00 - z01) / 2. * ood;
        dgy = (z01 + z11 - z00 - z10) / 2. * ood;
    }
    gx = (float)dgx;
    gy = (float)dgy;
    ct = (float)cos(atan(sqrt(dgx * dgx + dgy * dgy)));
}

struct PartIn {
    const double *x, *v, *vz, *h, *m;
};

struct Contrib {
    int ib, jb;
    float f[2];
    float q[SQ + 1];  // m, m vx, m vy, m h, m vz, K gx, K gy, K h / (2 dx)
};

__device__ __forceinline__ bool particle(const PartIn& P, int p, const double* z, int Nx, int Ny, double dx, float g, Contrib& c) {
    const double ood = 1.0 / dx;
    const double ux = P.x[2 * p] * ood, uy = P.x[2 * p + 1] * ood;
    c.ib = (int)floor(ux - 0.5);
    c.jb = (int)floor(uy - 0.5);
    c.f[0] = (float)(ux - c.ib);
    c.f[1] = (float)(uy - c.jb);
    if (c.ib < 0 || c.jb < 0 || c.ib + 2 > Nx - 1 || c.jb + 2 > Ny - 1) return false;
    float gx, gy, ct;
    cell_slope(z, Nx, Ny, ood, c.ib + (c.f[0] >= 1.f ? 1 : 0), c.jb + (c.f[1] >= 1.f ? 1 : 0), gx, gy, ct);
    const float m = (float)P.m[p], h = (float)P.h[p];
    const float K = m * g * ct * ct;
    c.q[0] = m;
    c.q[1] = m * (float)P.v[2 * p];
    c.q[2] = m * (float)P.v[2 * p + 1];
    c.q[3] = m * h;
    c.q[4] = m * (float)P.vz[p];
    c.q[5] = K * gx;
    c.q[6] = K * gy;
    c.q[7] = K * h * (float)(0.5 * ood);
    return true;
}

// pass 1: per-quantity bound of one contribution and particles per cell
__global__ void k_bounds(int* s, PartIn P, int Np, const double* z, int Nx, int Ny, double dx, float g, Box b) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < Np; p += gridDim.x * blockDim.x) {
        Contrib c;
        const bool ok = particle(P, p, z, Nx, Ny, dx, g, c);
        const int li = c.ib - b.i0, lj = c.jb - b.j0;
        if (!ok || li < 0 || lj < 0 || li + 2 >= b.nI || lj + 2 >= b.nJ) {
            atomicOr(&s[8], 1);
            continue;
        }
        const int n = atomicAdd(&s[HDR + li * b.nJ + lj], 1) + 1;
        atomicMax(&s[7], n);
        const float bF = c.q[7] + fmaxf(fabsf(c.q[5]), fabsf(c.q[6]));
        atomicMax((unsigned*)&s[0], __float_as_uint(c.q[0]));
        atomicMax((unsigned*)&s[1], __float_as_uint(fabsf(c.q[1])));
        atomicMax((unsigned*)&s[2], __float_as_uint(fabsf(c.q[2])));
        atomicMax((unsigned*)&s[3], __float_as_uint(c.q[3]));
        atomicMax((unsigned*)&s[4], __float_as_uint(bF));
        atomicMax((unsigned*)&s[5], __float_as_uint(bF));
        atomicMax((unsigned*)&s[6], __float_as_uint(fabsf(c.q[4])));
    }
}

// bits below one quantum kept by a lo word: a node adds at most 9 * s[7]
// contributions (9 cells, s[7] particles in the fullest), each lo part at
// most 2^(L-1) in magnitude, so L = 31 - ceil(log2(9 s[7])) (at most 20)
// keeps every lo sum below 2^30
__device__ __forceinline__ int lo_bits(const int* s) { return lo_bits_for(9 * s[7]); }

__device__ __forceinline__ float scale_of(const int* s, int q, float* inv) {
    const float bound = 9.f * (float)s[7] * 0.75f * __uint_as_float((unsigned)s[q]);
    int e = 0;
    if (bound > 0.f) {
        int E;
        frexpf(bound, &E);
        e = min(max(30 - E, -120), 120);
    }
    *inv = ldexpf(1.f, -e);
    return ldexpf(1.f, e);
}

// pass 2: quadratic B-spline P2G with the reference's 3e-3 weight cut-off
// (src/simulation.cpp:726-798), contributions added as int32 hi/lo pairs
__global__ void k_p2g(int* s, PartIn P, int Np, const double* z, int Nx, int Ny, double dx, float g, Box b) {
    float sc[SQ], inv;
    for (int q = 0; q < SQ; ++q) sc[q] = scale_of(s, q, &inv);
    const float lo_mul = ldexpf(1.f, lo_bits(s));
    int* hi = s + HDR + MAXN;
    int* lo = hi + (size_t)SQ * MAXN;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < Np; p += gridDim.x * blockDim.x) {
        Contrib c;
        if (!particle(P, p, z, Nx, Ny, dx, g, c)) continue;
        const int li = c.ib - b.i0, lj = c.jb - b.j0;
        if (li < 0 || lj < 0 || li + 2 >= b.nI || lj + 2 >= b.nJ) continue;
        float wx[3], wy[3], dwx[3], dwy[3];
        bspline3(c.f[0], wx, dwx);
        bspline3(c.f[1], wy, dwy);
        for (int a = 0; a < 3; ++a)
            for (int bb = 0; bb < 3; ++bb) {
                const float w = wx[a] * wy[bb];
                if (!(w > 3e-3f)) continue;
                const int nd = (li + a) * b.nJ + (lj + bb);
                const float v[SQ] = {c.q[0] * w, c.q[1] * w, c.q[2] * w, c.q[3] * w, c.q[7] * (dwx[a] * wy[bb]) - c.q[5] * w,
                                     c.q[7] * (dwy[bb] * wx[a]) - c.q[6] * w, c.q[4] * w};
                for (int q = 0; q < SQ; ++q) {
                    const float xs = v[q] * sc[q];
                    const int h_ = __float2int_rn(xs);
                    atomicAdd(&hi[(size_t)q * MAXN + nd], h_);
                    const int l_ = __float2int_rn((xs - (float)h_) * lo_mul);
                    if (l_) atomicAdd(&lo[(size_t)q * MAXN + nd], l_);
                }
            }
    }
}

// grid update with dt = 0 (computeGridVelocity of simulate()'s t=0 pass,
// src/simulation.cpp:493-495, 800-875): normalised h, v, vz and the mass
__global__ void k_grid(const int* s, Box b, double* out_h, double* out_m, double* out_v, double* out_vz) {
    float inv[SQ];
    for (int q = 0; q < SQ; ++q) scale_of(s, q, &inv[q]);
    const double lo_div = ldexp(1.0, -lo_bits(s));
    const int* hi = s + HDR + MAXN;
    const int* lo = hi + (size_t)SQ * MAXN;
    const int n = b.nI * b.nJ;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        float q[SQ];
        for (int r = 0; r < SQ; ++r)
            q[r] = (float)(((double)hi[(size_t)r * MAXN + k] + (double)lo[(size_t)r * MAXN + k] * lo_div) * (double)inv[r]);
        const float mi = q[0];
        float hn = 0.f, vzn = 0.f, vx = 0.f, vy = 0.f;
        if (mi > 1e-6f) {
            hn = q[3] / mi;
            vzn = q[6] / mi;
            const float vtx = q[1] / mi, vty = q[2] / mi;  // + dt * F / m with dt = 0
            if (vtx * vtx + vty * vty > 1e-16f) {
                vx = vtx;  // the friction decrement dt * a_f is zero at t = 0
                vy = vty;
            }
        }
        out_h[k] = hn;
        out_m[k] = mi;
        out_v[2 * k] = vx;
        out_v[2 * k + 1] = vy;
        out_vz[k] = vzn;
    }
}

std::mutex g_setup_mutex;
int* g_symbol_addr[64] = {nullptr};

}  // namespace
}  // namespace slab

using namespace slab;

extern "C" slab_status slab_initial_grid_static(const slab_terrain_desc* terrain, const double* d_z, const slab_params* params, int32_t Np,
                                               const double* d_x_xy, const double* d_v_xy, const double* d_vz, const double* d_h,
                                               const double* d_mass, const int32_t box[4], double* d_h_out, double* d_mass_out,
                                               double* d_v_out, double* d_vz_out, void* stream) {
    auto fail = [](slab_status st, const std::string& msg) {
        set_thread_error(msg);
        return st;
    };
    if (!terrain || !d_z || !params || !box || !d_x_xy || !d_v_xy || !d_vz || !d_h || !d_mass || !d_h_out || !d_mass_out || !d_v_out ||
        !d_vz_out)
        return fail(SLAB_E_ARG, "slab_initial_grid_static: null argument");
    if (Np < 0) return fail(SLAB_E_ARG, "slab_initial_grid_static: Np < 0");
    if (terrain->Nx < 3 || terrain->Ny < 3 || !(terrain->dx > 0.0))
        return fail(SLAB_E_ARG, "slab_initial_grid_static: terrain smaller than 3x3 nodes or dx <= 0");
    // extents in 64 bits: box values straight from the caller cannot overflow
    const int64_t nI64 = (int64_t)box[1] - box[0] + 1, nJ64 = (int64_t)box[3] - box[2] + 1;
    if (box[0] < 0 || box[2] < 0 || box[1] > terrain->Nx - 1 || box[3] > terrain->Ny - 1 || nI64 < 3 || nJ64 < 3)
        return fail(SLAB_E_ARG, "slab_initial_grid_static: box outside the terrain or smaller than 3x3 nodes");
    if (nI64 * nJ64 > SLAB_STATIC_MAX_NODES)
        return fail(SLAB_E_ARG, "slab_initial_grid_static: box has " + std::to_string(nI64 * nJ64) + " nodes, the maximum is " +
                                    std::to_string(SLAB_STATIC_MAX_NODES));
    const int nI = (int)nI64, nJ = (int)nJ64;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) return fail(SLAB_E_CUDA, "slab_initial_grid_static: no usable CUDA device");
    int* scratch = nullptr;
    {
        // once per device, with that device current: the device address of
        // the static array (its name is only a host-side stand-in)
        std::lock_guard<std::mutex> lk(g_setup_mutex);
        if (!g_symbol_addr[dev]) {
            e = cudaGetSymbolAddress(reinterpret_cast<void**>(&g_symbol_addr[dev]), g_scratch);
            if (e != cudaSuccess) {
                g_symbol_addr[dev] = nullptr;
                return fail(SLAB_E_CUDA, std::string("slab_initial_grid_static: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            }
        }
        scratch = g_symbol_addr[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const Box b{box[0], box[2], nI, nJ};
    const PartIn P{d_x_xy, d_v_xy, d_vz, d_h, d_mass};
    const float g = (float)params->gravity;
    const int pblocks = std::max(1, std::min((Np + 255) / 256, 148 * 8));
    const int nblocks = std::max(1, std::min((nI * nJ + 255) / 256, 148 * 8));
    k_clear<<<nblocks, 256, 0, st>>>(scratch, nI * nJ);
    k_bounds<<<pblocks, 256, 0, st>>>(scratch, P, Np, d_z, terrain->Nx, terrain->Ny, terrain->dx, g, b);
    k_p2g<<<pblocks, 256, 0, st>>>(scratch, P, Np, d_z, terrain->Nx, terrain->Ny, terrain->dx, g, b);
    k_grid<<<nblocks, 256, 0, st>>>(scratch, b, d_h_out, d_mass_out, d_v_out, d_vz_out);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(SLAB_E_CUDA, std::string("slab_initial_grid_static: launch: ") + cudaGetErrorString(e));
    int err = 0;
    e = cudaMemcpyAsync(&err, scratch + 8, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(SLAB_E_CUDA, std::string("slab_initial_grid_static: ") + cudaGetErrorString(e));
    if (err) return fail(SLAB_E_DOMAIN, "slab_initial_grid_static: a particle stencil lies outside the box or the terrain");
    return SLAB_OK;
}
