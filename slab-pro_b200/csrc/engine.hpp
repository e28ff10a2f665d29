// Host-side engine: the context behind the C ABI and the interface of the two
// step-loop implementations (plain FP64, split FP32).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <functional>
#include <map>
#include <memory>
#include <thread>
#include <string>
#include <vector>

#include "common.cuh"
#include "slab_gpu.h"

namespace slab {

// Thrown inside the library, turned into a slab_status at the C boundary.
struct Error {
    slab_status code;
    std::string msg;
};

#define SLAB_CUDA(call)                                                                                     \
    do {                                                                                                    \
        cudaError_t e_ = (call);                                                                            \
        if (e_ != cudaSuccess)                                                                              \
            throw ::slab::Error{e_ == cudaErrorMemoryAllocation ? SLAB_E_OOM : SLAB_E_CUDA,                 \
                                std::string(#call) + ": " + cudaGetErrorString(e_)};                        \
    } while (0)

template <typename T> T* dmalloc(size_t n) {
    void* p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc(&p, n * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error{SLAB_E_OOM, "cudaMalloc of " + std::to_string(n * sizeof(T)) + " bytes failed: " + cudaGetErrorString(e)};
    }
    return static_cast<T*>(p);
}

struct DFree {
    void operator()(void* p) const { cudaFree(p); }
};
template <typename T> using dptr = std::unique_ptr<T, DFree>;
template <typename T> dptr<T> dalloc(size_t n) { return dptr<T>(dmalloc<T>(n)); }

// Grow-only device scratch for the transient buffers of one call (binning an
// upload, building a download): kept at the largest size asked so far, so
// repeated calls allocate nothing. Callers finish their work on it (stream
// synchronised) before they return.
struct Scratch {
    dptr<char> buf;
    size_t cap = 0;
    char* get(size_t bytes) {
        if (bytes > cap) {
            buf.reset();  // cudaFree waits for the device: no work still uses the old buffer
            buf = dalloc<char>(bytes);
            cap = bytes;
        }
        return buf.get();
    }
};

// Carves 256-byte aligned pieces out of one scratch block.
struct Carve {
    size_t off = 0;
    template <typename T> size_t take(size_t n) {
        const size_t at = off;
        off += (n * sizeof(T) + 255) / 256 * 256;
        return at;
    }
};

// Runs f(begin, end) over [0, n) in up to 8 host threads (one for small n):
// for per-particle host work on millions of particles (input checks).
template <typename F> void parallel_ranges(int64_t n, F f) {
    const int64_t min_chunk = 1 << 18;
    const unsigned hw = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
    const int nt = (int)std::max<int64_t>(1, std::min<int64_t>(hw, n / min_chunk));
    if (nt <= 1) {
        f((int64_t)0, n);
        return;
    }
    std::vector<std::thread> th;
    const int64_t per = (n + nt - 1) / nt;
    for (int t = 0; t < nt; ++t) {
        const int64_t b = t * per, e = std::min(n, b + per);
        if (b < e) th.emplace_back([=] { f(b, e); });
    }
    for (auto& x : th) x.join();
}

// A grid download with no field pointer set only reports the box.
inline bool grid_view_wants_fields(const slab_grid_view& g) { return g.h || g.mass || g.v || g.vz || g.flip || g.F || g.a; }

// Grid::a = F / m_i where m_i > 1e-6, zero elsewhere, as computeGridVelocity
// leaves it (src/simulation.cpp:807-814; remesh zero-fills it, :626-627).
inline void fill_grid_acceleration(double* a, const double* F, const double* m, size_t n) {
    for (size_t k = 0; k < n; ++k) {
        const bool moving = m[k] > 1e-6;
        a[2 * k] = moving ? F[2 * k] / m[k] : 0.0;
        a[2 * k + 1] = moving ? F[2 * k + 1] / m[k] : 0.0;
    }
}

// Terrain metric terms shared by both paths, computed once on the device in
// FP64 (Simulation::terrainGradients / terrainTheta,
// src/complex_terrain.cpp:84-111).
struct Terrain {
    int Nx = 0, Ny = 0;
    double dx = 0, xll = 0, yll = 0;
    dptr<double> z;        // Nx*Ny
    dptr<double2> grad;    // cell gradient stored at the bottom-left node
    dptr<double> cos_t;    // cos(atan|grad|)
    dptr<float4> dem32;    // FP32 copy for the split path: gx, gy, cos(theta), z
};

// CUDA graphs of `chunk` consecutive steps, one per chunk size used.
struct StepGraphs {
    std::map<int, cudaGraphExec_t> g;
    ~StepGraphs() { clear(); }
    void clear() {
        for (auto& kv : g) cudaGraphExecDestroy(kv.second);
        g.clear();
    }
    void launch(int chunk, cudaStream_t st, const std::function<void()>& one_step) {
        auto it = g.find(chunk);
        if (it == g.end()) {
            cudaGraph_t gr;
            SLAB_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            for (int k = 0; k < chunk; ++k) one_step();
            SLAB_CUDA(cudaStreamEndCapture(st, &gr));
            cudaGraphExec_t ex;
            cudaError_t e = cudaGraphInstantiate(&ex, gr, 0);
            cudaGraphDestroy(gr);
            SLAB_CUDA(e);
            it = g.emplace(chunk, ex).first;
        }
        SLAB_CUDA(cudaGraphLaunch(it->second, st));
    }
};

// Per-kernel device times of profiled steps: events between the 4 kernels of
// each step, read back lazily. Phases: 0 begin/dt, 1 (unused: binning is
// fused into G2P), 2 P2G, 3 grid update, 4 G2P.
struct PhaseTimer {
    bool on = false;
    std::vector<cudaEvent_t> pool;
    std::vector<std::array<int, 6>> pending;
    size_t used = 0;
    double acc[5] = {0, 0, 0, 0, 0};
    int64_t steps = 0;
    ~PhaseTimer() {
        for (auto e : pool) cudaEventDestroy(e);
    }
    void reset() {
        pending.clear();
        used = 0;
        for (double& a : acc) a = 0;
        steps = 0;
    }
    int mark(cudaStream_t st) {
        if (used == pool.size()) {
            cudaEvent_t e;
            SLAB_CUDA(cudaEventCreate(&e));
            pool.push_back(e);
        }
        SLAB_CUDA(cudaEventRecord(pool[used], st));
        return (int)used++;
    }
    // the kernels of one step and the phase (out[] slot) each one counts to
    int nk = 4;
    int phase_of[5] = {0, 2, 3, 4, 0};
    // launches: nk callables, one per kernel of the step
    void profiled_step(cudaStream_t st, const std::function<void(int)>& launch_kernel) {
        std::array<int, 6> ev{};
        ev[0] = mark(st);
        for (int k = 0; k < nk; ++k) {
            launch_kernel(k);
            ev[k + 1] = mark(st);
        }
        pending.push_back(ev);
    }
    void collect() {
        if (pending.empty()) return;
        SLAB_CUDA(cudaEventSynchronize(pool[pending.back()[nk]]));
        for (auto& ev : pending) {
            for (int k = 0; k < nk; ++k) {
                float ms = 0;
                SLAB_CUDA(cudaEventElapsedTime(&ms, pool[ev[k]], pool[ev[k + 1]]));
                acc[phase_of[k]] += ms;
            }
            ++steps;
        }
        pending.clear();
        used = 0;
    }
};

struct Path {
    virtual ~Path() = default;
    virtual void upload(int Np, const double* x, const double* v, const double* vz, const double* h, const double* A, const double* m,
                        const double* z) = 0;
    virtual void initial_pass() = 0;
    // enqueue up to `chunk` steps; the device control block decides which run
    virtual void enqueue_steps(int chunk) = 0;
    // start an advance call on the device (budget, frame stop); false: the
    // caller arms the control block itself
    virtual bool arm(int64_t, int) { return false; }
    virtual void download_particles(double* x, double* v, double* vz, double* h, double* A, double* m, double* z) = 0;
    virtual void download_grid(slab_grid_view* view) = 0;
    virtual void download_max(double* h_max, double* v_max2) = 0;
    virtual void conservation(double out[4]) = 0;
    // FP64 particle moments: mass, centre of mass (x, y), momentum (x, y),
    // kinetic energy (moments.cuh)
    virtual void moments(double out[6]) = 0;
    // enqueue the packing of the current frame on the path's stream:
    // d_part Np x 8 float32 vertices (x y vx vy vz z h A, upload order),
    // d_grid 6 GeoTIFF bands over box {i0, i1, j0, j1} (slab_frame)
    virtual void pack_frame(float* d_part, float* d_grid, const int32_t box[4]) = 0;
    virtual int64_t launches() const = 0;
    virtual void phase_times(double out[5]) { for (int k = 0; k < 5; ++k) out[k] = 0; }
    virtual void set_profiling(bool) {}
    // CTA counts of the work kernels and tuning passes (the FP32 path's tuner)
    virtual void launch_shapes(int32_t out[6]) { for (int k = 0; k < 6; ++k) out[k] = 0; }
    // chunks of steps as one persistent cooperative launch (FP32_SPLIT)
    virtual void set_persistent(bool, long long) { throw Error{SLAB_E_ARG, "persistent steps need FP32_SPLIT"}; }
};

std::unique_ptr<Path> make_plain64(const Terrain& t, const slab_params& p, cudaStream_t s, Ctl* d_ctl, Ctl* h_ctl);
std::unique_ptr<Path> make_split32(const Terrain& t, const slab_params& p, cudaStream_t s, Ctl* d_ctl, Ctl* h_ctl);

void compute_terrain_metrics(Terrain& t, cudaStream_t s);

}  // namespace slab
