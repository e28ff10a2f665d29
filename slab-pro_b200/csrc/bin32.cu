// Device-side binning of a new FP32 split scenario: the particles a caller
// hands over in the reference layout (src/data_arrays.hpp:22-47, FP64, x and
// v interleaved) become the tile segments of particle buffer 0, sorted by
// tile and, inside a tile, in upload order -- the state every later step
// starts from. The reference keeps particles unsorted until its first
// block sort (src/simulation.cpp:540, 644-724); the split path bins them once,
// here, and keeps them binned in G2P.
//
// One upload of the raw arrays, then on the device: the split position and
// tile of every particle, a stable radix sort of (tile, upload index), the
// runs of equal tiles, and one gather into the segment layout. The host only
// reads back the occupied tiles (for the node-block reserve) and the particle
// box. Bitwise the same layout a host counting sort by tile would give.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_run_length_encode.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>

#include "bin32.hpp"

namespace slab {
namespace {

// Split position of particle q (src/simulation.cpp:741-742: i_base =
// int(x/dx - 0.5)), with the rounding written out so that no multiply-add is
// fused: the same bits as the same arithmetic on the host.
__global__ void k_bin_keys(int Np, const double* __restrict__ x, const double* __restrict__ v, double ood, double dx, int Nx, int Ny,
                           int TY, int32_t* __restrict__ cell, float2* __restrict__ f, uint32_t* __restrict__ key,
                           int32_t* __restrict__ val, unsigned long long* __restrict__ red) {
    // positions are >= 0 and speeds squared too: their bit patterns order like
    // the values, so the box and the speed bound reduce as integers -- per
    // thread, then per warp, then one atomic per warp and bound
    unsigned long long bx0 = 0x7ff0000000000000ull, bx1 = 0ull, by0 = 0x7ff0000000000000ull, by1 = 0ull, bv = 0ull;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < Np; q += gridDim.x * blockDim.x) {
        const double ux = __dmul_rn(x[2 * q], ood), uy = __dmul_rn(x[2 * q + 1], ood);
        int ib = (int)floor(__dsub_rn(ux, 0.5)), jb = (int)floor(__dsub_rn(uy, 0.5));
        float fx = (float)__dsub_rn(ux, (double)ib), fy = (float)__dsub_rn(uy, (double)jb);
        if (fx >= 1.5f) {
            ++ib;
            fx -= 1.f;
        }
        if (fy >= 1.5f) {
            ++jb;
            fy -= 1.f;
        }
        const bool inside = ib >= 0 && jb >= 0 && ib + 2 <= Nx - 1 && jb + 2 <= Ny - 1;
        if (!inside) {
            atomicOr(&red[5], 1ull);
            ib = min(max(ib, 0), Nx - 3);  // keeps the key in range; the call fails
            jb = min(max(jb, 0), Ny - 3);
        }
        cell[q] = pack_cell(ib, jb);
        f[q] = make_float2(fx, fy);
        key[q] = (uint32_t)((ib / TILE) * TY + (jb / TILE));
        val[q] = q;
        const double px = __dmul_rn(__dadd_rn((double)ib, (double)fx), dx), py = __dmul_rn(__dadd_rn((double)jb, (double)fy), dx);
        const float vx = (float)v[2 * q], vy = (float)v[2 * q + 1];
        const double vv = (double)__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy));
        const unsigned long long ux_ = (unsigned long long)__double_as_longlong(px), uy_ = (unsigned long long)__double_as_longlong(py);
        bx0 = min(bx0, ux_);
        bx1 = max(bx1, ux_);
        by0 = min(by0, uy_);
        by1 = max(by1, uy_);
        bv = max(bv, (unsigned long long)__double_as_longlong(vv));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        bx0 = min(bx0, __shfl_xor_sync(0xffffffffu, bx0, o));
        bx1 = max(bx1, __shfl_xor_sync(0xffffffffu, bx1, o));
        by0 = min(by0, __shfl_xor_sync(0xffffffffu, by0, o));
        by1 = max(by1, __shfl_xor_sync(0xffffffffu, by1, o));
        bv = max(bv, __shfl_xor_sync(0xffffffffu, bv, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&red[0], bx0);
        atomicMax(&red[1], bx1);
        atomicMin(&red[2], by0);
        atomicMax(&red[3], by1);
        atomicMax(&red[4], bv);
    }
}

// particle k of buffer 0 is upload index order[k]
__global__ void k_bin_gather(int Np, const int32_t* __restrict__ order, const int32_t* __restrict__ cell, const float2* __restrict__ f,
                             const double* __restrict__ v, const double* __restrict__ vz, const double* __restrict__ h,
                             const double* __restrict__ m, const double* __restrict__ z, PBuf out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < Np; k += gridDim.x * blockDim.x) {
        const int q = order[k];
        out.cell[k] = cell[q];
        out.f[k] = f[q];
        out.v[k] = make_float2((float)v[2 * q], (float)v[2 * q + 1]);
        out.h[k] = (float)h[q];
        out.m[k] = (float)m[q];
        out.vz[k] = (float)vz[q];
        out.z[k] = (float)z[q];
        out.id[k] = q;
    }
}

// segment record of occupied tile r (stamp 0) and its place on the first
// active list
__global__ void k_bin_records(int n, const uint32_t* __restrict__ tiles, const int32_t* __restrict__ counts,
                              const int32_t* __restrict__ starts, int32_t* grp, int32_t* act_list, int32_t* act_stamp) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const int t = (int)tiles[r];
        int32_t* G = grp + (size_t)t * GRP_STRIDE;
        for (int k = 0; k < GRP_STRIDE; ++k) G[k] = 0;
        G[0] = starts[r];
        G[1] = starts[r] + counts[r];
        G[2] = starts[r] + counts[r];
        G[3 + 4] = counts[r];
        G[GRP_STAMP] = 0;
        act_list[r] = t;
        act_stamp[t] = 0;
    }
}

// the caller's arrays may be host or device memory (a release generated on the device)
template <typename T> void cpy_h2d(T* d, const T* h, size_t n, cudaStream_t s) {
    if (n) SLAB_CUDA(cudaMemcpyAsync(d, h, n * sizeof(T), cudaMemcpyDefault, s));
}

}  // namespace

BinResult bin_particles(const Terrain& T, int TY, int ntiles, cudaStream_t st, int Np, const double* x, const double* v, const double* vz,
                        const double* h, const double* m, const double* z, const PBuf& out, int32_t* grp0, int32_t* act_list0,
                        int32_t* act_stamp, int act_cap, Scratch& scratch) {
    BinResult res;
    if (Np <= 0) return res;
    int end_bit = 1;
    while (end_bit < 32 && (1ll << end_bit) < (long long)ntiles) ++end_bit;
    // temporary bytes of the three library passes (size queries only)
    size_t t_sort = 0, t_rle = 0, t_scan = 0;
    SLAB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t_sort, (uint32_t*)nullptr, (uint32_t*)nullptr, (int32_t*)nullptr, (int32_t*)nullptr, Np,
                                              0, end_bit, st));
    SLAB_CUDA(cub::DeviceRunLengthEncode::Encode(nullptr, t_rle, (uint32_t*)nullptr, (uint32_t*)nullptr, (int32_t*)nullptr, (int32_t*)nullptr,
                                                 Np, st));
    SLAB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, t_scan, (int32_t*)nullptr, (int32_t*)nullptr, Np, st));
    size_t t_bytes = std::max<size_t>(1, std::max(t_sort, std::max(t_rle, t_scan)));
    // one scratch block: the raw arrays (x, v: 2 per particle; vz, h, m, z),
    // keys, values, runs and the library's temporary storage
    Carve cv;
    const size_t o_raw = cv.take<double>((size_t)8 * Np), o_cell = cv.take<int32_t>(Np), o_val = cv.take<int32_t>(Np),
                 o_val_s = cv.take<int32_t>(Np), o_f = cv.take<float2>(Np), o_key = cv.take<uint32_t>(Np), o_key_s = cv.take<uint32_t>(Np),
                 o_uniq = cv.take<uint32_t>(Np), o_counts = cv.take<int32_t>(Np), o_starts = cv.take<int32_t>(Np),
                 o_nruns = cv.take<int32_t>(1), o_red = cv.take<unsigned long long>(6), o_tmp = cv.take<char>(t_bytes);
    char* base = scratch.get(cv.off);
    double* dx_ = reinterpret_cast<double*>(base + o_raw);
    double* dv = dx_ + 2 * (size_t)Np;
    double* dvz = dv + 2 * (size_t)Np;
    double* dh = dvz + Np;
    double* dm = dh + Np;
    double* dz = dm + Np;
    int32_t* cell = reinterpret_cast<int32_t*>(base + o_cell);
    int32_t* val = reinterpret_cast<int32_t*>(base + o_val);
    int32_t* val_s = reinterpret_cast<int32_t*>(base + o_val_s);
    float2* f = reinterpret_cast<float2*>(base + o_f);
    uint32_t* key = reinterpret_cast<uint32_t*>(base + o_key);
    uint32_t* key_s = reinterpret_cast<uint32_t*>(base + o_key_s);
    uint32_t* uniq = reinterpret_cast<uint32_t*>(base + o_uniq);
    int32_t* counts = reinterpret_cast<int32_t*>(base + o_counts);
    int32_t* starts = reinterpret_cast<int32_t*>(base + o_starts);
    int32_t* nruns = reinterpret_cast<int32_t*>(base + o_nruns);
    unsigned long long* red = reinterpret_cast<unsigned long long*>(base + o_red);
    char* tmp = base + o_tmp;
    cpy_h2d(dx_, x, 2 * (size_t)Np, st);
    cpy_h2d(dv, v, 2 * (size_t)Np, st);
    cpy_h2d(dvz, vz, Np, st);
    cpy_h2d(dh, h, Np, st);
    cpy_h2d(dm, m, Np, st);
    cpy_h2d(dz, z, Np, st);
    const unsigned long long red0[6] = {0x7ff0000000000000ull, 0ull, 0x7ff0000000000000ull, 0ull, 0ull, 0ull};
    cpy_h2d(red, red0, 6, st);
    const int blocks = std::max(1, std::min((Np + 255) / 256, 148 * 16));
    k_bin_keys<<<blocks, 256, 0, st>>>(Np, dx_, dv, 1.0 / T.dx, T.dx, T.Nx, T.Ny, TY, cell, f, key, val, red);
    SLAB_CUDA(cudaGetLastError());
    SLAB_CUDA(cub::DeviceRadixSort::SortPairs(tmp, t_bytes, key, key_s, val, val_s, Np, 0, end_bit, st));
    SLAB_CUDA(cub::DeviceRunLengthEncode::Encode(tmp, t_bytes, key_s, uniq, counts, nruns, Np, st));
    int n = 0;
    unsigned long long hred[6];
    SLAB_CUDA(cudaMemcpyAsync(&n, nruns, sizeof(int), cudaMemcpyDeviceToHost, st));
    SLAB_CUDA(cudaMemcpyAsync(hred, red, sizeof(hred), cudaMemcpyDeviceToHost, st));
    SLAB_CUDA(cudaStreamSynchronize(st));
    if (hred[5]) throw Error{SLAB_E_DOMAIN, "particle stencil outside the terrain"};
    if (n > act_cap) throw Error{SLAB_E_OOM, "active tile capacity"};
    SLAB_CUDA(cub::DeviceScan::ExclusiveSum(tmp, t_bytes, counts, starts, n, st));
    k_bin_gather<<<blocks, 256, 0, st>>>(Np, val_s, cell, f, dv, dvz, dh, dm, dz, out);
    k_bin_records<<<std::max(1, std::min((n + 127) / 128, 148 * 8)), 128, 0, st>>>(n, uniq, counts, starts, grp0, act_list0, act_stamp);
    SLAB_CUDA(cudaGetLastError());
    res.tiles.resize(n);
    SLAB_CUDA(cudaMemcpyAsync(res.tiles.data(), uniq, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    SLAB_CUDA(cudaStreamSynchronize(st));  // the scratch is free again on return
    for (int k = 0; k < 4; ++k) res.box_bits[k] = hred[k];
    res.vmax2_bits = hred[4];
    return res;
}

}  // namespace slab
