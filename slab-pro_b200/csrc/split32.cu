// Host side of the FP32 split-precision step loop: per-scenario device
// storage, particle upload (binning into tiles), step launch / CUDA-graph
// capture, and downloads that restore the reference layouts.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <type_traits>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include "engine.hpp"
#include "engine32.hpp"
#include "split32_kernels.cuh"
#include "moments.cuh"
#include "bin32.hpp"

namespace slab {

namespace {
template <typename T> void h2d(T* d, const T* h, size_t n, cudaStream_t s) {
    if (n) SLAB_CUDA(cudaMemcpyAsync(d, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
}
template <typename T> void d2h(T* h, const T* d, size_t n, cudaStream_t s) {
    if (n) SLAB_CUDA(cudaMemcpyAsync(h, d, n * sizeof(T), cudaMemcpyDeviceToHost, s));
}

// Zeroes n doubles with up to 8 host threads: the maxima maps of a large
// terrain are hundreds of MB, mostly pages of the caller's arrays that were
// never touched, and one thread takes tens of milliseconds to fault them in.
void zero_fill(double* p, size_t n) {
    if (!p || n == 0) return;
    const unsigned hw = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
    if (n < ((size_t)1 << 20) || hw == 1) {
        std::memset(p, 0, n * sizeof(double));
        return;
    }
    const size_t per = (n + hw - 1) / hw;
    std::vector<std::thread> th;
    size_t done = 0;  // the prefix handed to threads
    try {
        for (unsigned k = 0; k < hw && done < n; ++k) {
            const size_t a = done, b = std::min(n, a + per);
            th.emplace_back([p, a, b] { std::memset(p + a, 0, (b - a) * sizeof(double)); });
            done = b;
        }
    } catch (const std::system_error&) {  // no thread to be had: the rest on this one
    }
    if (done < n) std::memset(p + done, 0, (n - done) * sizeof(double));
    for (auto& t : th) t.join();
}
}  // namespace

namespace k32 {

// Dense copies of per-block node fields for downloads: node (i, j) of the box
// [i0, i0+nI) x [j0, j0+nJ) reads the block of its owner tile if that block
// was updated at `stepid` (any stamp if stepid < 0), else 0.
__global__ void k_gather_nodes(const int32_t* __restrict__ blk_of, const int32_t* __restrict__ blk_stamp, int stepid, int TY, int i0,
                               int j0, int nI, int nJ, int nf, const float* const* __restrict__ fields, const float4* __restrict__ nv,
                               float* __restrict__ out) {
    const int64_t total = (int64_t)nI * nJ;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        const int i = i0 + (int)(k / nJ), j = j0 + (int)(k % nJ);
        const int blk = blk_of[(i / TILE) * TY + (j / TILE)];
        const bool ok = blk >= 0 && (stepid < 0 || blk_stamp[blk] == stepid);
        const size_t n = (size_t)blk * NCELL + (i % TILE) * TILE + (j % TILE);
        for (int q = 0; q < nf; ++q) out[q * total + k] = ok ? fields[q][n] : 0.f;
        if (nv) {  // velocity and FLIP increment
            const float4 v = ok ? nv[n] : make_float4(0.f, 0.f, 0.f, 0.f);
            out[nf * total + k] = v.x;
            out[(nf + 1) * total + k] = v.y;
            out[(nf + 2) * total + k] = v.z;
            out[(nf + 3) * total + k] = v.w;
        }
    }
}

// The whole-terrain max maps in FP64 (zero where the scenario's blocks never
// reached), for a download straight into page-locked caller memory.
__global__ void k_max_full(const int32_t* __restrict__ blk_of, int TY, int Nx, int Ny, const float* __restrict__ hmax,
                           const float* __restrict__ vmax2, double* __restrict__ oh, double* __restrict__ ov) {
    const int64_t total = (int64_t)Nx * Ny;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(k / Ny), j = (int)(k % Ny);
        const int blk = blk_of[(i / TILE) * TY + (j / TILE)];
        const size_t n = (size_t)blk * NCELL + (i % TILE) * TILE + (j % TILE);
        oh[k] = blk >= 0 ? (double)hmax[n] : 0.0;
        ov[k] = blk >= 0 ? (double)vmax2[n] : 0.0;
    }
}

// Frame packing (slab_frame_capture). Particle k of the buffer goes to vertex
// id[k]: x y vx vy vz z h A as float32 (the PLY vertex layout), A = m / (h rho).
__global__ void k_pack_particles(PBuf B, int Np, double dx, double rho, float* __restrict__ out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < Np; k += gridDim.x * blockDim.x) {
        const int32_t c = B.cell[k];
        const float2 f = B.f[k], v = B.v[k];
        const float h = B.h[k], m = B.m[k];
        float* o = out + (size_t)B.id[k] * 8;
        o[0] = (float)(((double)cell_i(c) + (double)f.x) * dx);
        o[1] = (float)(((double)cell_j(c) + (double)f.y) * dx);
        o[2] = v.x;
        o[3] = v.y;
        o[4] = B.vz[k];
        o[5] = B.z[k];
        o[6] = h;
        o[7] = (float)((double)m / ((double)h * rho));
    }
}

// Particle downloads in the reference layout (src/data_arrays.hpp:22-47):
// particle k of the buffer goes to index id[k] (upload order) of FP64 arrays;
// x = (cell + offset) dx and A = m / (h rho), each operation rounded as
// written. A null array is skipped; an id out of range raises *bad.
struct Unpack {
    double *x, *v, *vz, *h, *A, *m, *z;
};
__global__ void k_unpack_particles(PBuf B, int Np, double dx, double rho, Unpack o, int* __restrict__ bad) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < Np; k += gridDim.x * blockDim.x) {
        const int q = B.id[k];
        if ((unsigned)q >= (unsigned)Np) {
            atomicOr(bad, 1);
            continue;
        }
        const int32_t c = B.cell[k];
        const float2 f = B.f[k];
        if (o.x) {
            o.x[2 * q] = __dmul_rn(__dadd_rn((double)cell_i(c), (double)f.x), dx);
            o.x[2 * q + 1] = __dmul_rn(__dadd_rn((double)cell_j(c), (double)f.y), dx);
        }
        if (o.v) {
            const float2 v = B.v[k];
            o.v[2 * q] = v.x;
            o.v[2 * q + 1] = v.y;
        }
        if (o.vz) o.vz[q] = B.vz[k];
        if (o.h) o.h[q] = B.h[k];
        if (o.m) o.m[q] = B.m[k];
        if (o.A) o.A[q] = __ddiv_rn((double)B.m[k], __dmul_rn((double)B.h[k], rho));
        if (o.z) o.z[q] = B.z[k];
    }
}

// The grid box's 6 GeoTIFF bands (h, |v|, m, vx, vy, vz) in GDAL order:
// band-major, row 0 = the north edge (j = j0 + nJ - 1), x fastest; -9999 in
// every band where h == 0. Nodes of blocks the last step did not update are
// empty.
__global__ void k_pack_grid(const int32_t* __restrict__ blk_of, const int32_t* __restrict__ blk_stamp, int stepid, int TY, int i0, int j0,
                            int nI, int nJ, const float* __restrict__ oh, const float* __restrict__ om, const float* __restrict__ ovz,
                            const float4* __restrict__ nv, float* __restrict__ out) {
    const int64_t total = (int64_t)nI * nJ;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(k / nI), ci = (int)(k % nI);
        const int i = i0 + ci, j = j0 + nJ - 1 - r;
        const int blk = blk_of[(i / TILE) * TY + (j / TILE)];
        const bool ok = blk >= 0 && blk_stamp[blk] == stepid;
        const size_t n = (size_t)blk * NCELL + (i % TILE) * TILE + (j % TILE);
        const float h = ok ? oh[n] : 0.f;
        if (h == 0.f) {
            for (int q = 0; q < 6; ++q) out[q * total + k] = -9999.f;
            continue;
        }
        const float4 v = nv[n];
        out[k] = h;
        out[total + k] = (float)sqrt(__dadd_rn(__dmul_rn(v.x, v.x), __dmul_rn(v.y, v.y)));  // as the host writer: no fused multiply-add
        out[2 * total + k] = om[n];
        out[3 * total + k] = v.x;
        out[4 * total + k] = v.y;
        out[5 * total + k] = ovz[n];
    }
}

}  // namespace k32

void Engine32::pack_frame(int sid, float* d_part, float* d_grid, const int32_t box[4], double rho) {
    Store& S = (*slots[sid]);
    const SCnt c = counters(sid);
    const int b = c.seq & 1;
    const int Np = S.Np;
    if (!c.vz_valid) {  // between output frames the step loop does not keep z / vz
        k32::k_refresh_vz_z<<<std::max(1, std::min(148 * 8, (Np + 255) / 256)), 256, 0, st>>>(shared(), host_scn[sid].buf[b], Np, T.z.get());
        ++nlaunch;
    }
    k32::k_pack_particles<<<std::max(1, std::min(148 * 8, (Np + 255) / 256)), 256, 0, st>>>(host_scn[sid].buf[b], Np, T.dx, rho, d_part);
    const int nI = box[1] - box[0] + 1, nJ = box[3] - box[2] + 1;
    const int64_t nodes = (int64_t)nI * nJ;
    if (nodes > 0)
        k32::k_pack_grid<<<(int)std::max<int64_t>(1, std::min<int64_t>((nodes + 255) / 256, 148 * 8)), 256, 0, st>>>(
            S.blk_of.get(), d_blk_stamp.get(), c.stepid, TY, box[0], box[2], nI, nJ, d_oh.get(), d_om.get(), d_ovz.get(), d_nv.get(),
            d_grid);
    nlaunch += nodes > 0 ? 2 : 1;
    SLAB_CUDA(cudaGetLastError());
}

namespace {
// cuTensorMapEncodeTiled, found through the runtime (no link to the driver library)
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encode_tiled() {
    static EncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
        else
            cudaGetLastError();
    });
    return fn;
}
}  // namespace

Engine32::Engine32(const Terrain& t, cudaStream_t s, int max_scn, int64_t blk_cap, bool batch)
    : T(t), st(s), max_scn(max_scn), batch(batch) {
    TX = (t.Nx + TILE - 1) / TILE;
    TY = (t.Ny + TILE - 1) / TILE;
    ntiles = TX * TY;
    this->blk_cap = (int)std::min<int64_t>(blk_cap, INT32_MAX);
    d_nv = dalloc<float4>((size_t)this->blk_cap * NCELL);
    d_hmax = dalloc<float>((size_t)this->blk_cap * NCELL);
    d_vmax2 = dalloc<float>((size_t)this->blk_cap * NCELL);
    d_oh = dalloc<float>((size_t)this->blk_cap * NCELL);
    d_om = dalloc<float>((size_t)this->blk_cap * NCELL);
    d_ovz = dalloc<float>((size_t)this->blk_cap * NCELL);
    d_oFx = dalloc<float>((size_t)this->blk_cap * NCELL);
    d_oFy = dalloc<float>((size_t)this->blk_cap * NCELL);
    d_blk_stamp = dalloc<int32_t>(this->blk_cap);
    d_blk_owner = dalloc<int32_t>(this->blk_cap);
    d_misc = dalloc<int32_t>(8);
    d_work_pref = dalloc<int32_t>(max_scn + 1);
    d_scn = dalloc<Scn>(max_scn);
    d_cnt = dalloc<SCnt>(max_scn);
    h_cnt.resize(max_scn);
    slots.resize(max_scn);
    spare.resize(max_scn);
    d_collect = dalloc<int32_t>((size_t)ntiles + 8);
    d_free_blocks = dalloc<int32_t>(this->blk_cap);
    SLAB_CUDA(cudaMemsetAsync(d_hmax.get(), 0, (size_t)this->blk_cap * NCELL * sizeof(float), st));
    SLAB_CUDA(cudaMemsetAsync(d_vmax2.get(), 0, (size_t)this->blk_cap * NCELL * sizeof(float), st));
    SLAB_CUDA(cudaMemsetAsync(d_blk_stamp.get(), 0xff, (size_t)this->blk_cap * sizeof(int32_t), st));
    SLAB_CUDA(cudaMemsetAsync(d_misc.get(), 0, 8 * sizeof(int32_t), st));
    SLAB_CUDA(cudaMemsetAsync(d_work_pref.get(), 0, (max_scn + 1) * sizeof(int32_t), st));
    host_scn.resize(max_scn);
    SLAB_CUDA(cudaFuncSetAttribute(k32::k_p2g<k32::ACC_I32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(k32::P2GSmem)));
    SLAB_CUDA(cudaFuncSetAttribute(k32::k_p2g<k32::ACC_HILO>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(k32::P2GSmem)));
    SLAB_CUDA(cudaFuncSetAttribute(k32::k_p2g<k32::ACC_I64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(k32::P2GSmem)));
    SLAB_CUDA(cudaFuncSetAttribute(k32::k_p2g_cell<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(k32::P2CSmem)));
    SLAB_CUDA(cudaFuncSetAttribute(k32::k_p2g_cell<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(k32::P2CSmemTma)));
    if (const char* e = std::getenv("SLAB_P2G_TMA")) p2g_tma = std::atoi(e) != 0;
    {
        // the terrain window of the cell P2G as one tensor copy per tile: the
        // float4 terrain seen as [Nx][4 Ny] floats (rows 16 Ny bytes apart), boxes
        // of (TILE + 1) nodes by 4 (TILE + 1) floats (a multiple of 16 bytes);
        // boxes past the far edges read zeros
        const EncodeTiled enc = encode_tiled();
        if (!enc) throw Error{SLAB_E_CUDA, "cuTensorMapEncodeTiled is not available"};
        const cuuint64_t dims[2] = {(cuuint64_t)4 * T.Ny, (cuuint64_t)T.Nx};
        const cuuint64_t strides[1] = {(cuuint64_t)T.Ny * sizeof(float4)};
        const cuuint32_t box[2] = {4 * (TILE + 1), TILE + 1};
        const cuuint32_t estr[2] = {1, 1};
        const CUresult r = enc(&dem_map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void*)T.dem32.get(), dims, strides, box, estr,
                               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) throw Error{SLAB_E_CUDA, "cuTensorMapEncodeTiled failed for the terrain (code " + std::to_string((int)r) + ")"};
    }
    SLAB_CUDA(cudaFuncSetAttribute(k32::k_p2g_warp, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(k32::P2W_WARPS * sizeof(k32::P2WWarp))));
    if (const char* e = std::getenv("SLAB_P2G_ACC")) acc_mode = std::atoi(e);
    if (const char* e = std::getenv("SLAB_P2G_SPLIT")) split_min = std::atoi(e);
    split_min = std::min(split_min, k32::P2S_CAP);
    int dev = 0, sms = 0, occ_p = 0, occ_g = 0, occ_u = 0;
    SLAB_CUDA(cudaGetDevice(&dev));
    SLAB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    SLAB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_p, k32::k_p2g_warp, k32::P2W_THREADS,
                                                            k32::P2W_WARPS * sizeof(k32::P2WWarp)));
    int occ_c = 0, occ_h = 0;
    if (p2g_tma)
        SLAB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_c, k32::k_p2g_cell<true>, k32::P2C_THREADS, sizeof(k32::P2CSmemTma)));
    else
        SLAB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_c, k32::k_p2g_cell<false>, k32::P2C_THREADS, sizeof(k32::P2CSmem)));
    SLAB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_h, k32::k_p2g<k32::ACC_HILO>, k32::P2G_THREADS, sizeof(k32::P2GSmem)));
    SLAB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_g, k32::k_g2p, NCELL, 0));
    SLAB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_u, k32::k_grid, NCELL, 0));
    grid_p2g = sms * std::max(occ_p, 1);
    grid_p2g_cell = sms * std::max(occ_c, 1);
    grid_p2g_hilo = sms * std::max(occ_h, 1);
    int occ_s = 0;
    SLAB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_s, k32::k_p2g_sparse, k32::P2S_THREADS, sizeof(k32::P2SSmem)));
    grid_p2g_sparse = sms * std::max(occ_s, 1);
    grid_g2p = sms * std::max(occ_g, 1);
    grid_grid = sms * std::max(occ_u, 1);
    int occ_d = 0;
    SLAB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_d, k32::k_prep, 256, 0));
    grid_prep = sms * std::max(occ_d, 1);  // one resident wave, one thread per active tile
    const int base[Tuner::NK] = {grid_prep, grid_p2g_cell, grid_p2g_sparse, grid_grid, grid_g2p};
    std::copy(base, base + Tuner::NK, tune.base);
    if (const char* e = std::getenv("SLAB_TUNE")) tune.enabled = std::atoi(e) != 0;
    // the persistent step kernel: as many CTAs as can be resident at once
    // (a cooperative launch needs every CTA on the device together)
    int coop = 0, occ_ps = 0;
    SLAB_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    SLAB_CUDA(cudaFuncSetAttribute(k32::k_persist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k32::PERSIST_SMEM));
    SLAB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_ps, k32::k_persist, NCELL, k32::PERSIST_SMEM));
    grid_persist = coop ? sms * occ_ps : 0;
    if (const char* e = std::getenv("SLAB_PERSIST")) persist = std::atoi(e) != 0 && grid_persist > 0;
    timer.nk = 5;  // k_prep, P2G, grid update, G2P, k_end
    const int phase_map[5] = {1, 2, 3, 4, 0};
    for (int k = 0; k < 5; ++k) timer.phase_of[k] = phase_map[k];
}

Engine32::~Engine32() {}

Shared Engine32::shared() const {
    Shared sh{};
    sh.Nx = T.Nx;
    sh.Ny = T.Ny;
    sh.TX = TX;
    sh.TY = TY;
    sh.dem = T.dem32.get();
    sh.nv = d_nv.get();
    sh.hmax = d_hmax.get();
    sh.vmax2 = d_vmax2.get();
    sh.oh = d_oh.get();
    sh.om = d_om.get();
    sh.ovz = d_ovz.get();
    sh.oFx = d_oFx.get();
    sh.oFy = d_oFy.get();
    sh.blk_stamp = d_blk_stamp.get();
    sh.blk_owner = d_blk_owner.get();
    sh.blk_count = d_misc.get();
    sh.blk_cap = blk_cap;
    sh.nscn = nscn;
    sh.scn = d_scn.get();
    sh.cnt = d_cnt.get();
    sh.work_pref = d_work_pref.get();
    sh.wlist = d_wlist.get();
    sh.wcount = d_misc.get() + 2;
    sh.split_min = acc_mode == k32::ACC_MIXED ? split_min : -1;
    sh.gflat = d_gflat.get();
    sh.gcount = d_misc.get() + 6;
    sh.gcap = 4 * work_cap;
    sh.desc = d_desc.get();
    sh.part = d_part.get();
    sh.work_cap = work_cap;
    sh.free_blocks = d_free_blocks.get();
    sh.free_count = d_misc.get() + 4;
    return sh;
}

namespace k32 {
// node blocks of one scenario: ids into out[8...], count into out[0], tile
// box {ti0, ti1, tj0, tj1} into out[1..4] (out[0..4] preset to 0, big, -1, big, -1)
__global__ void k_collect_blocks(const int32_t* __restrict__ blk_of, int ntiles, int TY, int32_t* out) {
    const int lane = threadIdx.x & 31;
    for (int t0 = blockIdx.x * blockDim.x; t0 < ntiles; t0 += gridDim.x * blockDim.x) {
        const int t = t0 + threadIdx.x;
        const int b = t < ntiles ? blk_of[t] : -1;
        const unsigned m = __ballot_sync(0xffffffffu, b >= 0);
        if (!m) continue;
        int base = 0;
        if (lane == __ffs(m) - 1) base = atomicAdd(out, __popc(m));
        base = __shfl_sync(0xffffffffu, base, __ffs(m) - 1);
        if (b >= 0) {
            out[8 + base + __popc(m & ((1u << lane) - 1u))] = b;
            atomicMin(out + 1, t / TY);
            atomicMax(out + 2, t / TY);
            atomicMin(out + 3, t % TY);
            atomicMax(out + 4, t % TY);
        }
    }
}

__global__ void k_release_blocks(const int32_t* ids, int n, float* hmax, float* vmax2, int32_t* stamp, int32_t* owner) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < (int64_t)n * NCELL; k += (int64_t)gridDim.x * blockDim.x) {
        const int b = ids[k / NCELL];
        const size_t e = (size_t)b * NCELL + (k % NCELL);
        hmax[e] = 0.f;
        vmax2[e] = 0.f;
        if (k % NCELL == 0) {
            stamp[b] = -1;
            owner[b] = -1;
        }
    }
}
}  // namespace k32

void Engine32::retire(int sid, const Ctl& empty_ctl) {
    if (sid < 0 || sid >= nscn || !slots[sid]) throw Error{SLAB_E_NOTFOUND, "no scenario in this slot"};
    Store& S = *slots[sid];
    int tb[4];
    const int nblk = collect_blocks(sid, tb);  // ids in d_collect[8...], on the device
    if (nblk > 0) {
        int32_t free_count = 0;
        d2h(&free_count, d_misc.get() + 4, 1, st);
        SLAB_CUDA(cudaStreamSynchronize(st));
        const int32_t* ids = d_collect.get() + 8;
        const int blocks = (int)std::min<int64_t>(((int64_t)nblk * NCELL + 255) / 256, 148 * 8);
        k32::k_release_blocks<<<blocks, 256, 0, st>>>(ids, nblk, d_hmax.get(), d_vmax2.get(), d_blk_stamp.get(), d_blk_owner.get());
        SLAB_CUDA(cudaGetLastError());
        SLAB_CUDA(cudaMemcpyAsync(d_free_blocks.get() + free_count, ids, (size_t)nblk * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
        const int32_t nf = free_count + nblk;
        h2d(d_misc.get() + 4, &nf, 1, st);
        SLAB_CUDA(cudaStreamSynchronize(st));
    }
    // an empty slot: a stopped control block and no tiles
    SCnt zero{};
    h2d(S.cnt, &zero, 1, st);
    h2d(S.ctl, &empty_ctl, 1, st);
    Scn D = Scn{};
    D.ctl = S.ctl;
    D.cnt = S.cnt;
    h2d(d_scn.get() + sid, &D, 1, st);
    host_scn[sid] = D;
    work_cap_total -= S.act_cap;
    SLAB_CUDA(cudaStreamSynchronize(st));
    spare[sid] = std::move(slots[sid]);
    free_slots.push_back(sid);
}

int Engine32::collect_blocks(int sid, int tbox[4]) {
    Store& S = *slots[sid];
    const int32_t init[5] = {0, INT32_MAX, -1, INT32_MAX, -1};
    h2d(d_collect.get(), init, 5, st);
    const int blocks = (int)std::min<int64_t>(((int64_t)ntiles + 255) / 256, 148 * 8);
    k32::k_collect_blocks<<<blocks, 256, 0, st>>>(S.blk_of.get(), ntiles, TY, d_collect.get());
    SLAB_CUDA(cudaGetLastError());
    int32_t res[5];
    d2h(res, d_collect.get(), 5, st);
    SLAB_CUDA(cudaStreamSynchronize(st));
    for (int k = 0; k < 4; ++k) tbox[k] = res[1 + k];
    return res[0];
}

void Engine32::box_of_blocks(int sid, int box[4]) {
    int tb[4];
    if (collect_blocks(sid, tb) == 0) {
        box[0] = box[2] = 0;
        box[1] = box[3] = -1;
        return;
    }
    box[0] = tb[0] * TILE;
    box[1] = std::min(T.Nx - 1, tb[1] * TILE + TILE - 1);
    box[2] = tb[2] * TILE;
    box[3] = std::min(T.Ny - 1, tb[3] * TILE + TILE - 1);
}

void Engine32::download_max_box(int sid, const int box[4], double* hmax, double* vmax2) {
    const int nI = box[1] - box[0] + 1, nJ = box[3] - box[2] + 1;
    if (nI <= 0 || nJ <= 0) return;
    const std::vector<float> f = gather_nodes(sid, -1, box[0], box[2], nI, nJ, {d_hmax.get(), d_vmax2.get()}, false);
    const size_t n = (size_t)nI * nJ;
    for (size_t k = 0; k < n; ++k) {
        if (hmax) hmax[k] = f[k];
        if (vmax2) vmax2[k] = f[n + k];
    }
}

void Engine32::ensure_work_cap(int64_t need) {
    if (need <= work_cap) return;
    const int64_t cap = std::min<int64_t>(std::max<int64_t>(need, (int64_t)work_cap * 3 / 2), INT32_MAX / PART_STRIDE);
    SLAB_CUDA(cudaStreamSynchronize(st));
    d_desc = dalloc<TileDesc>(cap);
    d_part = dalloc<float>((size_t)cap * PART_STRIDE);
    d_gflat = dalloc<int32_t>((size_t)8 * cap);  // up to 4 grid tiles per active tile, 2 ints each
    d_wlist = dalloc<int32_t>((size_t)2 * cap);
    work_cap = (int)cap;
    graphs.clear();
}

int Engine32::add_scenario(const slab_params& p, Ctl* ctl, Ctl* h_ctl, int Np, const double* x, const double* v, const double* vz,
                           const double* h, const double* m, const double* z, int want_slot) {
    int sid;
    if (want_slot >= 0) {
        auto it = std::find(free_slots.begin(), free_slots.end(), want_slot);
        if (it != free_slots.end()) {
            free_slots.erase(it);
        } else if (want_slot == nscn && nscn < max_scn) {
        } else {
            throw Error{SLAB_E_STATE, "scenario slot is not free"};
        }
        sid = want_slot;
        // slots between the high-water mark and want_slot would stay unused: not allowed
        if (sid > nscn) throw Error{SLAB_E_STATE, "scenario slots must be filled in order"};
    } else if (!free_slots.empty()) {
        sid = free_slots.back();
        free_slots.pop_back();
    } else {
        if (nscn >= max_scn) throw Error{SLAB_E_OOM, "scenario capacity exceeded"};
        sid = nscn;
    }
    // a retired scenario's arrays stay with its slot and are reused: the
    // terrain-sized tile arrays always, particle buffers and tile lists when
    // large enough (admission then allocates nothing in the common case)
    if (spare[sid]) slots[sid] = std::move(spare[sid]);
    else slots[sid].reset(new Store());
    Store& S = *slots[sid];
    S.Np = Np;
    S.ctl = ctl;
    S.h_ctl = h_ctl;
    // a single scenario gets the safe bound; in a batch the lists start at an
    // estimate (>= 4 particles per active tile) and grow between chunks
    S.act_cap = batch ? std::max(1, std::min(ntiles, Np / 4 + 256)) : std::max(1, std::min(ntiles, Np));
    const bool new_parts = S.Np_alloc < Np, new_lists = S.act_alloc < S.act_cap, new_tiles = !S.blk_of;
    for (int b = 0; b < 2; ++b) {
        if (new_parts) {
            // padded past Np: P2G's bulk copies round a range's end up to 16 bytes
            S.cell[b] = dalloc<int32_t>(Np + PARTICLE_PAD);
            S.f[b] = dalloc<float2>(Np + PARTICLE_PAD);
            S.v[b] = dalloc<float2>(Np + PARTICLE_PAD);
            S.h[b] = dalloc<float>(Np + PARTICLE_PAD);
            S.m[b] = dalloc<float>(Np + PARTICLE_PAD);
            S.id[b] = dalloc<int32_t>(Np + PARTICLE_PAD);
            S.vz[b] = dalloc<float>(Np + PARTICLE_PAD);
            S.z[b] = dalloc<float>(Np + PARTICLE_PAD);
        }
        if (new_tiles) S.grp[b] = dalloc<int32_t>((size_t)ntiles * GRP_STRIDE);
        if (new_lists) S.act_list[b] = dalloc<int32_t>(S.act_cap);
    }
    if (new_parts) S.Np_alloc = Np;
    if (new_lists) S.act_alloc = S.act_cap;
    else S.act_cap = S.act_alloc;  // a reused list keeps its full length
    if (new_tiles) {
        S.act_stamp = dalloc<int32_t>(ntiles);
        S.slot_of = dalloc<int32_t>(ntiles);
        S.nxt_off = dalloc<int32_t>(ntiles);
        S.gt_stamp = dalloc<int32_t>(ntiles);
        S.blk_of = dalloc<int32_t>(ntiles);
    }
    S.cnt = d_cnt.get() + sid;
    ensure_work_cap(work_cap_total + S.act_cap);
    work_cap_total += S.act_cap;

    // ---- bin the particles into tile segments on the device (stable in upload order)
    const double ood = 1.0 / T.dx;
    for (int b = 0; b < 2; ++b)  // every record stale (stamp -1)
        SLAB_CUDA(cudaMemsetAsync(S.grp[b].get(), 0xff, (size_t)ntiles * GRP_STRIDE * sizeof(int32_t), st));
    SLAB_CUDA(cudaMemsetAsync(S.act_stamp.get(), 0xff, ntiles * sizeof(int32_t), st));
    const PBuf out0{S.cell[0].get(), S.f[0].get(), S.v[0].get(), S.h[0].get(), S.m[0].get(), S.id[0].get(), S.vz[0].get(), S.z[0].get()};
    const BinResult bin = bin_particles(T, TY, ntiles, st, Np, x, v, vz, h, m, z, out0, S.grp[0].get(), S.act_list[0].get(),
                                        S.act_stamp.get(), S.act_cap, scratch);
    const std::vector<uint32_t>& alist = bin.tiles;
    // node blocks the t=0 pass will take (the grid tiles of the active tiles'
    // node windows): grow the pool now, as the pass runs before any check
    {
        std::vector<char> touched(ntiles, 0);
        int64_t est = 0;
        for (uint32_t t : alist)
            for (int k = 0; k < 4; ++k) {
                const int gi = (int)t / TY + (k >> 1), gj = (int)t % TY + (k & 1);
                if (gi < TX && gj < TY && !touched[gi * TY + gj]) {
                    touched[gi * TY + gj] = 1;
                    ++est;
                }
            }
        int32_t misc[8];
        d2h(misc, d_misc.get(), 8, st);
        SLAB_CUDA(cudaStreamSynchronize(st));
        pending_blocks += est;
        const int64_t need = (int64_t)(misc[0] - misc[4]) + pending_blocks;
        if (2 * need > blk_cap) grow_blocks((int)std::min<int64_t>(std::max<int64_t>(2 * (int64_t)blk_cap, 2 * need), INT32_MAX / NCELL));
    }
    SLAB_CUDA(cudaMemsetAsync(S.gt_stamp.get(), 0xff, ntiles * sizeof(int32_t), st));
    SLAB_CUDA(cudaMemsetAsync(S.blk_of.get(), 0xff, ntiles * sizeof(int32_t), st));
    SCnt c0{};
    c0.act_count[0] = (int)alist.size();
    c0.t0_pending = 1;
    c0.vz_valid = 1;
    h2d(S.cnt, &c0, 1, st);
    // particle box and max speed for the first step (Simulation::updateDt / remesh)
    for (int k = 0; k < 4; ++k) h_ctl->pos_acc[k] = bin.box_bits[k];
    h_ctl->vmax2_bits = bin.vmax2_bits;
    h2d(ctl, h_ctl, 1, st);

    Scn& D = host_scn[sid];
    D = Scn{};
    D.ctl = ctl;
    D.cnt = S.cnt;
    D.g = (float)p.gravity;
    D.rho = (float)p.rho;
    D.fr = (float)p.flip_ratio;
    D.ood = (float)ood;
    D.fric = p.friction.type;
    D.mu_c = (float)p.friction.coulomb_mu;
    D.mu_v = (float)p.friction.voellmy_mu;
    D.xi = (float)p.friction.voellmy_xi;
    D.mu1 = (float)p.friction.mu_1;
    D.mu2 = (float)p.friction.mu_2;
    D.I0 = (float)p.friction.I0;
    D.d = (float)p.friction.d;
    D.phi = (float)p.friction.phi;
    D.Np = Np;
    for (int b = 0; b < 2; ++b) {
        D.buf[b] = PBuf{S.cell[b].get(), S.f[b].get(), S.v[b].get(), S.h[b].get(), S.m[b].get(), S.id[b].get(), S.vz[b].get(), S.z[b].get()};
        D.grp[b] = S.grp[b].get();
        D.act_list[b] = S.act_list[b].get();
    }
    D.act_stamp = S.act_stamp.get();
    D.slot_of = S.slot_of.get();
    D.nxt_off = S.nxt_off.get();
    D.gt_stamp = S.gt_stamp.get();
    D.blk_of = S.blk_of.get();
    D.act_cap = S.act_cap;
    h2d(d_scn.get() + sid, &D, 1, st);
    if (sid == nscn) {
        nscn += 1;
        graphs.clear();  // the step graphs carry the scenario count
    }
    return sid;
}

void Engine32::launch_begin(int t0) {
    k32::k_begin<<<1, 1024, 0, st>>>(shared(), t0);
    SLAB_CUDA(cudaGetLastError());
}

void Engine32::launch_t0() {
    const Shared sh = shared();
    k32::k_begin<<<1, 1024, 0, st>>>(sh, 1);
    k32::k_prep<<<grid_prep, 256, 0, st>>>(sh);
    launch_p2g(sh);
    k32::k_grid<<<grid_grid, NCELL, 0, st>>>(sh);
    SLAB_CUDA(cudaGetLastError());
    nlaunch += acc_mode == k32::ACC_MIXED ? 5 : 4;
    pending_blocks = 0;  // later reads of the pool count see these blocks
}

// the cell-sorted P2G; SLAB_P2G_TMA=1 stages the next tile's loads with TMA
// bulk copies (same sums, in the same order)
void Engine32::launch_p2g_cell(const Shared& sh, int cls) {
    if (p2g_tma)
        k32::k_p2g_cell<true><<<grid_p2g_cell, k32::P2C_THREADS, sizeof(k32::P2CSmemTma), st>>>(sh, cls, dem_map);
    else
        k32::k_p2g_cell<false><<<grid_p2g_cell, k32::P2C_THREADS, sizeof(k32::P2CSmem), st>>>(sh, cls, dem_map);
}

void Engine32::launch_p2g(const Shared& sh) {
    if (acc_mode == k32::ACC_MIXED) {  // dense tiles, then sparse tiles
        launch_p2g_cell(sh, 0);
        k32::k_p2g_sparse<<<grid_p2g_sparse, k32::P2S_THREADS, sizeof(k32::P2SSmem), st>>>(sh, 1);
    } else if (acc_mode == k32::ACC_WARP) {
        k32::k_p2g_warp<<<grid_p2g, k32::P2W_THREADS, k32::P2W_WARPS * sizeof(k32::P2WWarp), st>>>(sh, -1);
    } else if (acc_mode == k32::ACC_CELL) {
        launch_p2g_cell(sh, -1);
    } else if (acc_mode == k32::ACC_I32) {
        k32::k_p2g<k32::ACC_I32><<<grid_p2g_hilo, k32::P2G_THREADS, sizeof(k32::P2GSmem), st>>>(sh, -1);
    } else if (acc_mode == k32::ACC_I64) {
        k32::k_p2g<k32::ACC_I64><<<grid_p2g_hilo, k32::P2G_THREADS, sizeof(k32::P2GSmem), st>>>(sh, -1);
    } else {
        k32::k_p2g<k32::ACC_HILO><<<grid_p2g_hilo, k32::P2G_THREADS, sizeof(k32::P2GSmem), st>>>(sh, -1);
    }
}

void Engine32::launch_kernel(int k, const Shared& sh) {
    switch (k) {
        case 0: k32::k_prep<<<grid_prep, 256, 0, st>>>(sh); break;
        case 1: launch_p2g(sh); break;
        case 2: k32::k_grid<<<grid_grid, NCELL, 0, st>>>(sh); break;
        case 3: k32::k_g2p<<<grid_g2p, NCELL, 0, st>>>(sh, T.z.get()); break;
        case 4: k32::k_end<<<1, 1024, 0, st>>>(sh); break;
    }
}

void Engine32::arm(int64_t steps_left, int stop_at_frame) {
    k32::k_arm_begin<<<1, 1024, 0, st>>>(shared(), steps_left, stop_at_frame);
    SLAB_CUDA(cudaGetLastError());
    nlaunch += 1;
}

void Engine32::launch_step() {
    const Shared sh = shared();
    for (int k = 0; k < 5; ++k) launch_kernel(k, sh);
}

constexpr int Engine32::Tuner::FACTOR4[];


namespace {
// Launch shapes picked for single scenarios, by device, tile count and
// particle count (half-octave buckets), kept for the process: a later context
// of the same size starts from them instead of measuring its first steps
// again. Shapes never change results, only time.
std::mutex g_tune_mu;
std::map<std::string, std::vector<int>> g_tune_cache;
}  // namespace

void Engine32::tune_key_for(int Np) {
    int dev = 0;
    SLAB_CUDA(cudaGetDevice(&dev));
    const int bucket = Np > 0 ? (int)std::floor(2.0 * std::log2((double)Np)) : 0;
    tune.key = std::to_string(dev) + ":" + std::to_string(TILE) + ":" + std::to_string(ntiles) + ":" + std::to_string(bucket);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    const auto it = g_tune_cache.find(tune.key);
    if (it == g_tune_cache.end() || !tune.enabled) return;
    std::copy(it->second.begin(), it->second.end(), tune.pick);
    apply_shapes(tune.pick);
    graphs.clear();
    tune.from_cache = true;
    tune.next = 256;  // no schedule on the first steps; the usual cadence after them
}

int Engine32::tuned_grid(int k, int c) const {
    if (tune.fixed[k] > 0) return tune.fixed[k];
    return std::max(1, tune.base[k] * Tuner::FACTOR4[c] / 4);
}

void Engine32::apply_shapes(const int* c) {
    int* g[Tuner::NK] = {&grid_prep, &grid_p2g_cell, &grid_p2g_sparse, &grid_grid, &grid_g2p};
    for (int k = 0; k < Tuner::NK; ++k) *g[k] = tuned_grid(k, c[k]);
}

void Engine32::launch_shapes(int out[5]) const {
    const int g[Tuner::NK] = {grid_prep, grid_p2g_cell, grid_p2g_sparse, grid_grid, grid_g2p};
    for (int k = 0; k < Tuner::NK; ++k) out[k] = g[k];
}

void Engine32::fix_shapes(const int32_t* grids, bool tune_on) {
    for (int k = 0; k < Tuner::NK; ++k) tune.fixed[k] = grids ? std::max<int32_t>(grids[k], 0) : 0;
    tune.enabled = tune_on;
    if (tune.state == 1) tune.state = 0;  // a schedule in flight is dropped (its events are not read)
    apply_shapes(tune.pick);
    graphs.clear();
}

// One MIXED step with an event before each kernel and after the last.
void Engine32::launch_step_timed(const Shared& sh, cudaEvent_t* e) {
    SLAB_CUDA(cudaEventRecord(e[0], st));
    k32::k_prep<<<grid_prep, 256, 0, st>>>(sh);
    SLAB_CUDA(cudaEventRecord(e[1], st));
    launch_p2g_cell(sh, 0);
    SLAB_CUDA(cudaEventRecord(e[2], st));
    k32::k_p2g_sparse<<<grid_p2g_sparse, k32::P2S_THREADS, sizeof(k32::P2SSmem), st>>>(sh, 1);
    SLAB_CUDA(cudaEventRecord(e[3], st));
    k32::k_grid<<<grid_grid, NCELL, 0, st>>>(sh);
    SLAB_CUDA(cudaEventRecord(e[4], st));
    k32::k_g2p<<<grid_g2p, NCELL, 0, st>>>(sh, T.z.get());
    SLAB_CUDA(cudaEventRecord(e[5], st));
    k32::k_end<<<1, 1024, 0, st>>>(sh);
    SLAB_CUDA(cudaEventRecord(e[6], st));
}

// Reads the schedule's events and keeps, per kernel, the candidate with the
// least summed time; the occupancy grid (candidate 2) stays unless another is
// faster by more than 3 %, so timing noise does not flip the shapes.
void Engine32::tune_pick() {
    constexpr int W = Tuner::NK + 2;
    SLAB_CUDA(cudaEventSynchronize(tune.ev[Tuner::NSTEP * W - 1]));
    double ms[Tuner::NK][Tuner::NC] = {};
    for (int s = 0; s < Tuner::NSTEP; ++s) {
        const int c = s % Tuner::NC;
        for (int k = 0; k < Tuner::NK; ++k) {
            float t = 0;
            SLAB_CUDA(cudaEventElapsedTime(&t, tune.ev[s * W + k], tune.ev[s * W + k + 1]));
            ms[k][c] += t;
        }
    }
    for (int k = 0; k < Tuner::NK; ++k) {
        int best = 2;
        for (int c = 0; c < Tuner::NC; ++c)
            if (ms[k][c] < 0.97 * ms[k][2] && ms[k][c] < ms[k][best]) best = c;
        tune.pick[k] = best;
    }
    apply_shapes(tune.pick);
    graphs.clear();  // the step graphs carry the grid sizes
    if (!tune.key.empty()) {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[tune.key] = std::vector<int>(tune.pick, tune.pick + Tuner::NK);
    }
    tune.state = 0;
    tune.tunes += 1;
    tune.next = std::max<int64_t>(4 * tune.steps, tune.steps + 256);
}

void Engine32::set_persistent(bool on, long long limit_cycles) {
    if (on && grid_persist <= 0) throw Error{SLAB_E_ARG, "this device cannot run a cooperative launch"};
    if (!on && persist && d_bar) {  // back to separate kernels: only from a complete step state
        k32::GridBar b{};
        d2h(&b, reinterpret_cast<k32::GridBar*>(d_bar.get()), 1, st);
        SLAB_CUDA(cudaStreamSynchronize(st));
        if (b.dead) dead = true;
    }
    if (on && acc_mode != k32::ACC_MIXED) throw Error{SLAB_E_ARG, "persistent steps run the default P2G scheme only"};
    persist = on;
    if (limit_cycles > 0) persist_limit = limit_cycles;
}

// One cooperative launch of k_persist for `chunk` steps. The barrier state
// starts from zero at every launch (a launch whose waits ran out leaves it
// anywhere).
void Engine32::launch_persistent(int chunk) {
    if (!d_bar) {
        d_bar = dalloc<unsigned>(sizeof(k32::GridBar) / sizeof(unsigned));
        SLAB_CUDA(cudaMemsetAsync(d_bar.get(), 0, sizeof(k32::GridBar), st));
    }
    SLAB_CUDA(cudaMemsetAsync(d_bar.get(), 0, 2 * sizeof(unsigned), st));  // count and generation; `dead` stays
    Shared sh = shared();
    const double* z64 = T.z.get();
    int n = chunk;
    long long lim = persist_limit;
    k32::GridBar* bar = reinterpret_cast<k32::GridBar*>(d_bar.get());
    void* args[] = {&sh, &z64, &n, &lim, &bar, &dem_map};
    SLAB_CUDA(cudaLaunchCooperativeKernel((const void*)k32::k_persist, dim3(grid_persist), dim3(NCELL), args, k32::PERSIST_SMEM, st));
    nlaunch += 1;
}

void Engine32::enqueue_steps(int chunk) {
    if (persist && d_bar && timer.on) {  // profiled steps run the separate kernels: only from a complete step state
        k32::GridBar b{};
        d2h(&b, reinterpret_cast<k32::GridBar*>(d_bar.get()), 1, st);
        SLAB_CUDA(cudaStreamSynchronize(st));
        if (b.dead) dead = true;
    }
    if (dead) throw Error{SLAB_E_TIMEOUT, "an earlier persistent launch gave up at a barrier; the step state is incomplete"};
    if (persist && acc_mode == k32::ACC_MIXED && !timer.on) {
        launch_persistent(chunk);
        tune.steps += chunk;
        return;
    }
    if (graph_nscn != nscn) {
        graphs.clear();
        graph_nscn = nscn;
    }
    int k = 0;
    if (tune.enabled && acc_mode == k32::ACC_MIXED && !timer.on) {
        if (tune.state == 2) tune_pick();
        const bool moved = tune.active > 0 && tune.active_at > 0 && (tune.active > 2 * tune.active_at || 2 * tune.active < tune.active_at);
        if (tune.state == 0 && nscn > 0 && (tune.steps >= tune.next || moved)) {
            constexpr int W = Tuner::NK + 2;
            while ((int)tune.ev.size() < Tuner::NSTEP * W) {
                cudaEvent_t e;
                SLAB_CUDA(cudaEventCreate(&e));
                tune.ev.push_back(e);
            }
            tune.state = 1;
            tune.done = 0;
            tune.active_at = std::max<int64_t>(tune.active, 1);
        }
        if (tune.state == 1) {
            const Shared sh = shared();
            for (; k < chunk && tune.done < Tuner::NSTEP; ++k, ++tune.done) {
                int c[Tuner::NK];
                for (int q = 0; q < Tuner::NK; ++q) c[q] = tune.done % Tuner::NC;
                apply_shapes(c);
                launch_step_timed(sh, tune.ev.data() + (size_t)tune.done * (Tuner::NK + 2));
            }
            apply_shapes(tune.pick);
            for (; k < chunk; ++k) launch_step();
            SLAB_CUDA(cudaGetLastError());
            if (tune.done == Tuner::NSTEP) tune.state = 2;
        }
    }
    if (k < chunk) {
        if (timer.on) {
            const Shared sh = shared();
            for (; k < chunk; ++k) timer.profiled_step(st, [&](int kk) { launch_kernel(kk, sh); });
            SLAB_CUDA(cudaGetLastError());
        } else {
            graphs.launch(chunk, st, [&] { launch_step(); });
        }
    }
    tune.steps += chunk;
    nlaunch += (acc_mode == k32::ACC_MIXED ? 6 : 5) * (int64_t)chunk;
}

SCnt Engine32::counters(int sid) {
    SCnt c;
    d2h(&c, (*slots[sid]).cnt, 1, st);
    SLAB_CUDA(cudaStreamSynchronize(st));
    return c;
}

bool Engine32::check_capacity() {
    if (!nscn) return false;
    d2h(h_cnt.data(), d_cnt.get(), nscn, st);
    int32_t used_blocks = 0;
    d2h(&used_blocks, d_misc.get(), 1, st);
    SLAB_CUDA(cudaStreamSynchronize(st));
    bool grew = false;
    int64_t active = 0;
    for (int s = 0; s < nscn; ++s) {
        if (!slots[s]) continue;
        const int need = std::max(h_cnt[s].act_count[0], h_cnt[s].act_count[1]);
        active += need;
        Store& S = (*slots[s]);
        if (2 * need > S.act_cap && S.act_cap < ntiles) {
            const int cap = std::min(ntiles, std::max(2 * S.act_cap, 4 * need));
            for (int b = 0; b < 2; ++b) {
                dptr<int32_t> nl = dalloc<int32_t>(cap);
                SLAB_CUDA(cudaMemcpyAsync(nl.get(), S.act_list[b].get(), S.act_cap * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
                S.act_list[b] = std::move(nl);
                host_scn[s].act_list[b] = S.act_list[b].get();
            }
            work_cap_total += cap - S.act_cap;
            S.act_cap = cap;
            S.act_alloc = cap;
            host_scn[s].act_cap = cap;
            h2d(d_scn.get() + s, &host_scn[s], 1, st);
            grew = true;
        }
    }
    tune.active = active;
    if (grew) ensure_work_cap(work_cap_total);
    if (2 * (int64_t)used_blocks > blk_cap) {
        grow_blocks((int)std::min<int64_t>((int64_t)blk_cap * 2, INT32_MAX / NCELL));
        grew = true;
    }
    if (grew) SLAB_CUDA(cudaStreamSynchronize(st));
    return grew;
}

void Engine32::grow_blocks(int cap) {
    if (cap <= blk_cap) return;
    auto grow = [&](auto& p, size_t per, int fill) {
        using E = typename std::remove_reference<decltype(*p.get())>::type;
        auto np = dalloc<E>((size_t)cap * per);
        SLAB_CUDA(cudaMemsetAsync(np.get(), fill, (size_t)cap * per * sizeof(E), st));
        SLAB_CUDA(cudaMemcpyAsync(np.get(), p.get(), (size_t)blk_cap * per * sizeof(E), cudaMemcpyDeviceToDevice, st));
        p = std::move(np);
    };
    grow(d_nv, NCELL, 0);
    grow(d_hmax, NCELL, 0);
    grow(d_vmax2, NCELL, 0);
    grow(d_oh, NCELL, 0);
    grow(d_om, NCELL, 0);
    grow(d_ovz, NCELL, 0);
    grow(d_oFx, NCELL, 0);
    grow(d_oFy, NCELL, 0);
    grow(d_blk_stamp, 1, 0xff);
    grow(d_blk_owner, 1, 0xff);
    grow(d_free_blocks, 1, 0);
    blk_cap = cap;
    graphs.clear();
}

void Engine32::download_particles(int sid, double* x, double* v, double* vz, double* h, double* A, double* m, double* z, double rho) {
    Store& S = (*slots[sid]);
    const SCnt c = counters(sid);
    const int b = c.seq & 1;
    const int Np = S.Np;
    if (!c.vz_valid && (vz || z)) {
        // between output frames the step loop does not keep z / vz
        k32::k_refresh_vz_z<<<std::min(148 * 8, (Np + 255) / 256), 256, 0, st>>>(shared(), host_scn[sid].buf[b], Np, T.z.get());
        SLAB_CUDA(cudaGetLastError());
    }
    if (Np <= 0) return;
    // the reference layout is built on the device, then each requested array
    // is one copy into the caller's memory (full link speed when it is pinned)
    double* const host[7] = {x, v, vz, h, A, m, z};
    const int width[7] = {2, 2, 1, 1, 1, 1, 1};
    size_t need = 0;
    for (int a = 0; a < 7; ++a)
        if (host[a]) need += (size_t)width[a] * Np;
    if (need == 0) return;
    double* const buf = reinterpret_cast<double*>(scratch.get(need * sizeof(double)));
    double* dev[7] = {};
    size_t off = 0;
    for (int a = 0; a < 7; ++a)
        if (host[a]) {
            dev[a] = buf + off;
            off += (size_t)width[a] * Np;
        }
    if (!d_unpack_bad) d_unpack_bad = dalloc<int32_t>(1);
    SLAB_CUDA(cudaMemsetAsync(d_unpack_bad.get(), 0, sizeof(int32_t), st));
    const k32::Unpack o{dev[0], dev[1], dev[2], dev[3], dev[4], dev[5], dev[6]};
    k32::k_unpack_particles<<<std::max(1, std::min(148 * 8, (Np + 255) / 256)), 256, 0, st>>>(host_scn[sid].buf[b], Np, T.dx, rho, o,
                                                                                        d_unpack_bad.get());
    SLAB_CUDA(cudaGetLastError());
    for (int a = 0; a < 7; ++a)
        if (host[a]) d2h(host[a], dev[a], (size_t)width[a] * Np, st);
    int32_t bad = 0;
    d2h(&bad, d_unpack_bad.get(), 1, st);
    SLAB_CUDA(cudaStreamSynchronize(st));
    if (bad) throw Error{SLAB_E_CUDA, "corrupt particle id"};
}

std::vector<float> Engine32::gather_nodes(int sid, int stepid, int i0, int j0, int nI, int nJ, const std::vector<const float*>& fields,
                                          bool with_v) {
    Store& S = (*slots[sid]);
    const int64_t total = (int64_t)nI * nJ;
    const int nout = (int)fields.size() + (with_v ? 4 : 0);
    std::vector<float> host((size_t)nout * total);
    if (total == 0) return host;
    // scratch kept between calls (downloads at every retirement must not allocate)
    if ((size_t)nout * total > gather_cap) {
        d_gather = dalloc<float>((size_t)nout * total);
        gather_cap = (size_t)nout * total;
    }
    if (!d_gather_fp) d_gather_fp = dalloc<const float*>(8);
    if (fields.size() > 8) throw Error{SLAB_E_ARG, "too many fields"};
    h2d(d_gather_fp.get(), fields.data(), fields.size(), st);
    const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 8);
    k32::k_gather_nodes<<<blocks, 256, 0, st>>>(S.blk_of.get(), d_blk_stamp.get(), stepid, TY, i0, j0, nI, nJ, (int)fields.size(),
                                                d_gather_fp.get(), with_v ? d_nv.get() : nullptr, d_gather.get());
    SLAB_CUDA(cudaGetLastError());
    d2h(host.data(), d_gather.get(), host.size(), st);
    SLAB_CUDA(cudaStreamSynchronize(st));
    return host;
}

void Engine32::download_grid(int sid, slab_grid_view* gv) {
    Store& S = (*slots[sid]);
    d2h(S.h_ctl, S.ctl, 1, st);
    const SCnt c = counters(sid);
    const int i0 = S.h_ctl->box[0], i1 = S.h_ctl->box[1], j0 = S.h_ctl->box[2], j1 = S.h_ctl->box[3];
    const int gNx = i1 - i0 + 1, gNy = j1 - j0 + 1;
    gv->Nx = gNx;
    gv->Ny = gNy;
    gv->i_off = i0;
    gv->j_off = j0;
    if (!grid_view_wants_fields(*gv)) return;  // box only
    if ((int64_t)gNx * gNy > gv->cap_nodes) throw Error{SLAB_E_ARG, "grid view capacity too small"};
    const std::vector<float> f =
        gather_nodes(sid, c.stepid, i0, j0, gNx, gNy, {d_oh.get(), d_om.get(), d_ovz.get(), d_oFx.get(), d_oFy.get()}, true);
    const size_t n = (size_t)gNx * gNy;
    const float *fh = f.data(), *fm = fh + n, *fvz = fm + n, *fFx = fvz + n, *fFy = fFx + n, *fvx = fFy + n, *fvy = fvx + n,
                *flx = fvy + n, *fly = flx + n;
    for (size_t k = 0; k < n; ++k) {
        if (gv->h) gv->h[k] = fh[k];
        if (gv->mass) gv->mass[k] = fm[k];
        if (gv->vz) gv->vz[k] = fvz[k];
        if (gv->v) {
            gv->v[2 * k] = fvx[k];
            gv->v[2 * k + 1] = fvy[k];
        }
        if (gv->flip) {
            gv->flip[2 * k] = flx[k];
            gv->flip[2 * k + 1] = fly[k];
        }
        if (gv->F) {
            gv->F[2 * k] = fFx[k];
            gv->F[2 * k + 1] = fFy[k];
        }
        if (gv->a) {  // the FP32 quotient of the grid update, F / m (src/simulation.cpp:814)
            const bool moving = fm[k] > 1e-6f;
            gv->a[2 * k] = moving ? (double)(fFx[k] / fm[k]) : 0.0;
            gv->a[2 * k + 1] = moving ? (double)(fFy[k] / fm[k]) : 0.0;
        }
    }
}

namespace {
bool page_locked(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}
}  // namespace

void Engine32::download_max(int sid, double* hmax, double* vmax2) {
    const size_t nn = (size_t)T.Nx * T.Ny;
    if (hmax && vmax2 && page_locked(hmax) && page_locked(vmax2)) {
        // page-locked destinations: the whole maps are built on the device and
        // each is one copy at full link speed (a host-side zero fill of the
        // untouched nodes would run at host memory speed instead)
        double* buf = reinterpret_cast<double*>(scratch.get(2 * nn * sizeof(double)));
        const int blocks = (int)std::min<int64_t>(((int64_t)nn + 255) / 256, 148 * 16);
        k32::k_max_full<<<blocks, 256, 0, st>>>((*slots[sid]).blk_of.get(), TY, T.Nx, T.Ny, d_hmax.get(), d_vmax2.get(), buf, buf + nn);
        SLAB_CUDA(cudaGetLastError());
        d2h(hmax, buf, nn, st);
        d2h(vmax2, buf + nn, nn, st);
        SLAB_CUDA(cudaStreamSynchronize(st));
        return;
    }
    // nodes outside the box of the scenario's node blocks were never updated:
    // zero; only the box is gathered on the device and copied back
    int box[4];
    box_of_blocks(sid, box);
    zero_fill(hmax, nn);
    zero_fill(vmax2, nn);
    const int nI = box[1] - box[0] + 1, nJ = box[3] - box[2] + 1;
    if (nI <= 0 || nJ <= 0) return;
    const std::vector<float> f = gather_nodes(sid, -1, box[0], box[2], nI, nJ, {d_hmax.get(), d_vmax2.get()}, false);
    const size_t n = (size_t)nI * nJ;
    for (int i = 0; i < nI; ++i) {
        const size_t row = (size_t)(box[0] + i) * T.Ny + box[2], src = (size_t)i * nJ;
        for (int j = 0; j < nJ; ++j) {
            if (hmax) hmax[row + j] = f[src + j];
            if (vmax2) vmax2[row + j] = f[n + src + j];
        }
    }
}

void Engine32::conservation(int sid, double out[4], double rho) {
    Store& S = (*slots[sid]);
    std::vector<double> v(2 * (size_t)S.Np), m(S.Np);
    download_particles(sid, nullptr, v.data(), nullptr, nullptr, nullptr, m.data(), nullptr, rho);
    double M = 0, Px = 0, Py = 0;
    for (int q = 0; q < S.Np; ++q) {
        M += m[q];
        Px += m[q] * v[2 * q];
        Py += m[q] * v[2 * q + 1];
    }
    const SCnt c = counters(sid);
    out[0] = M;
    out[1] = c.grid_mass;
    out[2] = Px;
    out[3] = Py;
}

namespace {
// position (from the split cell + offset), velocity and mass of particle p of
// a buffer, for the moments reduction
struct SplitParticle {
    const int32_t* cell;
    const float2* f;
    const float2* v;
    const float* m;
    double dx;
    __device__ void operator()(int p, double& x, double& y, double& vx, double& vy, double& mass) const {
        const int32_t c = cell[p];
        const float2 fp = f[p], vp = v[p];
        x = ((double)cell_i(c) + (double)fp.x) * dx;
        y = ((double)cell_j(c) + (double)fp.y) * dx;
        vx = vp.x;
        vy = vp.y;
        mass = m[p];
    }
};
}  // namespace

void Engine32::moments(int sid, double out[6]) {
    Store& S = (*slots[sid]);
    const SCnt c = counters(sid);
    const int b = c.seq & 1;  // the buffer the last G2P wrote
    if (!d_mom) d_mom = dalloc<double>((size_t)MOM_BLOCKS * MOM_N + MOM_N);
    const SplitParticle get{S.cell[b].get(), S.f[b].get(), S.v[b].get(), S.m[b].get(), T.dx};
    k_moments<<<MOM_BLOCKS, MOM_THREADS, 0, st>>>(S.Np, get, d_mom.get());
    k_moments_final<<<1, MOM_THREADS, 0, st>>>(d_mom.get(), d_mom.get() + (size_t)MOM_BLOCKS * MOM_N);
    nlaunch += 2;
    SLAB_CUDA(cudaGetLastError());
    d2h(out, d_mom.get() + (size_t)MOM_BLOCKS * MOM_N, MOM_N, st);
    SLAB_CUDA(cudaStreamSynchronize(st));
}

namespace {

// The single-scenario FP32 path behind slab_ctx.
struct Split32 final : Path {
    Engine32 E;
    slab_params prm;
    Ctl* dc;
    Ctl* hc;
    int sid = -1;
    Split32(const Terrain& t, const slab_params& p, cudaStream_t s, Ctl* d, Ctl* h)
        : E(t, s, 1, (int64_t)((t.Nx + TILE - 1) / TILE) * ((t.Ny + TILE - 1) / TILE)), prm(p), dc(d), hc(h) {}
    void upload(int Np, const double* x, const double* v, const double* vz, const double* h, const double* A, const double* m,
                const double* z) override {
        (void)A;
        sid = E.add_scenario(prm, dc, hc, Np, x, v, vz, h, m, z);
        E.tune_key_for(Np);
    }
    void initial_pass() override { E.launch_t0(); }
    void enqueue_steps(int chunk) override { E.enqueue_steps(chunk); }
    bool arm(int64_t steps_left, int stop_at_frame) override {
        E.arm(steps_left, stop_at_frame);
        return true;
    }
    void download_particles(double* x, double* v, double* vz, double* h, double* A, double* m, double* z) override {
        E.download_particles(sid, x, v, vz, h, A, m, z, prm.rho);
    }
    void download_grid(slab_grid_view* gv) override { E.download_grid(sid, gv); }
    void download_max(double* hm, double* vm) override { E.download_max(sid, hm, vm); }
    void conservation(double out[4]) override { E.conservation(sid, out, prm.rho); }
    void moments(double out[6]) override { E.moments(sid, out); }
    void pack_frame(float* d_part, float* d_grid, const int32_t box[4]) override { E.pack_frame(sid, d_part, d_grid, box, prm.rho); }
    int64_t launches() const override { return E.nlaunch; }
    void set_profiling(bool on) override {
        E.timer.collect();
        E.timer.reset();
        E.timer.on = on;
    }
    void phase_times(double out[5]) override {
        E.timer.collect();
        for (int k = 0; k < 5; ++k) out[k] = E.timer.acc[k];
    }
    void launch_shapes(int32_t out[6]) override {
        int g[5];
        E.launch_shapes(g);
        for (int k = 0; k < 5; ++k) out[k] = g[k];
        out[5] = E.tune.tunes;
    }
    void set_persistent(bool on, long long limit_cycles) override { E.set_persistent(on, limit_cycles); }
};

}  // namespace

std::unique_ptr<Path> make_split32(const Terrain& t, const slab_params& p, cudaStream_t s, Ctl* d_ctl, Ctl* h_ctl) {
    return std::unique_ptr<Path>(new Split32(t, p, s, d_ctl, h_ctl));
}

}  // namespace slab

#ifdef SLAB_PHASE_CLOCKS
// per-phase cycle sums of the P2G kernel (instrumented builds only); reading clears them
extern "C" int slab_debug_phase_clocks(unsigned long long* out16) {
    if (cudaMemcpyFromSymbol(out16, slab::k32::g_phase_clk, 16 * sizeof(unsigned long long)) != cudaSuccess) return 1;
    const unsigned long long z[16] = {0};
    return cudaMemcpyToSymbol(slab::k32::g_phase_clk, z, sizeof(z)) == cudaSuccess ? 0 : 1;
}
#endif
