// Shared device helpers and the per-scenario control block.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "slab_gpu.h"

namespace slab {

// Error bits a kernel may raise in Ctl::err; the host maps them to statuses.
enum : int32_t { ERR_DOMAIN = 1, ERR_NONFINITE = 2, ERR_MOVE = 4, ERR_CAPACITY = 8, ERR_TIMEOUT = 16 };

// Per-scenario control block in device memory. Time, dt and the frame logic
// live here so that many steps can run (or be replayed from a CUDA graph)
// without the host in the loop; see Simulation::simulate/updateDt
// (src/simulation.cpp:484-582).
struct Ctl {
    // parameters (copied from slab_params at upload)
    double dx, one_over_dx, C_cfl, dt_max, output_dt, total_time;
    // state
    double time;          // simulated time after the last completed step
    double dt;            // dt of the current / last step
    double new_time;      // time + dt of the current step
    int64_t steps;        // completed steps
    int64_t steps_left;   // budget of the running advance call
    int32_t frame;        // completed frames
    int32_t stop;         // 1: the running advance call is over; kernels skip
    int32_t active;       // 1: the current step runs
    int32_t frame_end;    // 1: the current step lands on an output frame
    int32_t stop_at_frame;
    int32_t frame_hit;    // set when a step completed a frame
    int32_t err;          // ERR_* bits
    int32_t write_outputs;  // grid output fields are written this step
    uint64_t vmax2_bits;  // max |v_p|^2 over particles after the last G2P (double bits; values >= 0)
    uint64_t vmax2_acc;   // accumulator of the running G2P
    // Particle bounding box (double bits of min x, max x, min y, max y; all
    // positions are >= 0 inside the terrain, so the bit patterns order like
    // the values). pos is the box at the start of the current step, pos_acc
    // collects the box after the running G2P.
    uint64_t pos[4];
    uint64_t pos_acc[4];
    // The reference's remeshed grid box for the current step
    // (src/simulation.cpp:602-612): nodes [box[0], box[1]] x [box[2], box[3]].
    int32_t box[4];
    uint32_t done_blocks;  // last-block-done counter
    int32_t keep_outputs;  // write grid output fields every step (tests); else frame steps only
    unsigned long long node_steps;  // grid nodes with mass > 1e-6, summed over all steps so far
};

// The reference's remesh box from the particle bounding box
// (src/simulation.cpp:602-606). Terrain node 0 sits at coordinate 0.
__host__ __device__ inline void remesh_box(double min_x, double max_x, double min_y, double max_y, double dx, double one_over_dx,
                                           int32_t box[4]) {
    const double epsilon = 1e-8 * dx;
    box[0] = (int32_t)(min_x * one_over_dx - 1.0 - epsilon);
    box[1] = (int32_t)(max_x * one_over_dx + 2.0 + epsilon);
    box[2] = (int32_t)(min_y * one_over_dx - 1.0 - epsilon);
    box[3] = (int32_t)(max_y * one_over_dx + 2.0 + epsilon);
}

// Quadratic B-spline and its derivative (src/tools.hpp:119-140), written for
// the three stencil nodes of a particle with in-cell offset f = x/dx - i_base
// in [0.5, 1.5): node distances f, f-1, f-2.
template <typename R> __device__ __forceinline__ void bspline3(R f, R w[3], R dw[3]) {
    const R a = R(1.5) - f;   // distance-based form of node 0: 0.5 (1.5 - |u|)^2, |u| = f
    const R b = f - R(1.0);   // node 1: |u| < 0.5
    const R c = f - R(0.5);   // node 2: 0.5 (1.5 - |u|)^2, |u| = 2 - f
    w[0] = R(0.5) * a * a;
    w[1] = R(0.75) - b * b;
    w[2] = R(0.5) * c * c;
    dw[0] = f - R(1.5);
    dw[1] = R(-2.0) * b;
    dw[2] = c;
}

// FP32: every operation rounded as written (no multiply-add contraction), so
// each kernel that evaluates the weights gets the same bits whatever code the
// compiler schedules around it.
template <> __device__ __forceinline__ void bspline3<float>(float f, float w[3], float dw[3]) {
    const float a = __fsub_rn(1.5f, f), b = __fsub_rn(f, 1.0f), c = __fsub_rn(f, 0.5f);
    w[0] = __fmul_rn(__fmul_rn(0.5f, a), a);
    w[1] = __fsub_rn(0.75f, __fmul_rn(b, b));
    w[2] = __fmul_rn(__fmul_rn(0.5f, c), c);
    dw[0] = __fsub_rn(f, 1.5f);
    dw[1] = __fmul_rn(-2.0f, b);
    dw[2] = c;
}

// Fixed-point P2G sums keep each contribution as an int32 pair: hi, the
// contribution rounded to the quantum, and lo, the rest below the quantum in
// units of 2^-L quanta (|lo| <= 2^(L-1)). With at most n contributions to a
// node, L = min(20, 31 - ceil(log2 n)) keeps every lo sum below 2^30 for any
// n, so no int32 sum can overflow however many particles share a cell.
__host__ __device__ inline int lo_bits_for(int n) {
    int c = 0;
    while (c < 31 && (1 << c) < n) ++c;  // ceil(log2 n), 0 for n <= 1
    const int L = 31 - c;
    return L < 20 ? L : 20;
}

__device__ __forceinline__ void atomic_max_u64(uint64_t* a, uint64_t v) {
    atomicMax(reinterpret_cast<unsigned long long*>(a), static_cast<unsigned long long>(v));
}

}  // namespace slab

namespace slab {

// Start of a step, one thread: the stop conditions of the running advance
// call, then Simulation::updateDt (src/simulation.cpp:565-582) from the
// previous G2P's max |v|^2, then the reference's remesh box from the
// particle bounding box (src/simulation.cpp:594-612). Products that feed a
// sum are rounded explicitly so no fused multiply-add changes the result.
__device__ inline void ctl_begin(Ctl* c, int Nx, int Ny) {
    c->active = 0;
    if (c->stop) return;
    if (c->steps_left <= 0 || !(c->time < c->total_time) || (c->stop_at_frame && c->frame_hit) || c->err) {
        c->stop = 1;
        return;
    }
    const double vmax2 = __longlong_as_double((long long)c->vmax2_bits);
    const double max_speed = sqrt(vmax2);
    double dt;
    if (max_speed > 0.0) {
        const double a = __dmul_rn(c->C_cfl, c->dx) / max_speed;
        dt = (c->dt_max < a) ? c->dt_max : a;  // std::min(a, dt_max)
    } else {
        dt = c->dt_max;
    }
    const double next_frame_time = __dmul_rn(c->output_dt, (double)(c->frame + 1));
    if (__dadd_rn(c->time, dt) > next_frame_time - 1e-12) dt = next_frame_time - c->time;
    c->dt = dt;
    c->new_time = __dadd_rn(c->time, dt);
    c->frame_end = (next_frame_time - c->new_time < 1e-13) ? 1 : 0;
    c->write_outputs = (c->frame_end || c->keep_outputs) ? 1 : 0;
    for (int k = 0; k < 4; ++k) c->pos[k] = c->pos_acc[k];
    remesh_box(__longlong_as_double((long long)c->pos[0]), __longlong_as_double((long long)c->pos[1]),
               __longlong_as_double((long long)c->pos[2]), __longlong_as_double((long long)c->pos[3]), c->dx, c->one_over_dx, c->box);
    if (c->box[0] < 0 || c->box[2] < 0 || c->box[1] > Nx - 1 || c->box[3] > Ny - 1) {
        c->err |= ERR_DOMAIN;
        c->stop = 1;
        return;
    }
    c->pos_acc[0] = 0x7ff0000000000000ull;  // +inf
    c->pos_acc[1] = 0;
    c->pos_acc[2] = 0x7ff0000000000000ull;
    c->pos_acc[3] = 0;
    c->vmax2_acc = 0;
    c->done_blocks = 0;
    c->active = 1;
}

// End of a step, one thread (the last block of G2P): time += dt and the frame
// bump of simulate() (src/simulation.cpp:503-505).
__device__ inline void ctl_end(Ctl* c) {
    c->time = c->new_time;
    c->steps += 1;
    c->steps_left -= 1;
    c->vmax2_bits = c->vmax2_acc;
    if (c->frame_end) {
        c->frame += 1;
        c->frame_hit = 1;
    }
}

// Same as ctl_begin for simulate()'s t=0 pass: dt = 0, no time advance.
__device__ inline void ctl_begin_t0(Ctl* c, int Nx, int Ny) {
    c->active = 0;
    c->dt = 0.0;
    c->new_time = c->time;
    c->frame_end = 0;
    c->write_outputs = 1;
    for (int k = 0; k < 4; ++k) c->pos[k] = c->pos_acc[k];
    remesh_box(__longlong_as_double((long long)c->pos[0]), __longlong_as_double((long long)c->pos[1]),
               __longlong_as_double((long long)c->pos[2]), __longlong_as_double((long long)c->pos[3]), c->dx, c->one_over_dx, c->box);
    if (c->box[0] < 0 || c->box[2] < 0 || c->box[1] > Nx - 1 || c->box[3] > Ny - 1) {
        c->err |= ERR_DOMAIN;
        return;
    }
    c->active = 1;
}

template <typename T> __device__ __forceinline__ T warp_max(T v) {
    for (int o = 16; o > 0; o >>= 1) {
        T w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}
template <typename T> __device__ __forceinline__ T warp_min(T v) {
    for (int o = 16; o > 0; o >>= 1) {
        T w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}

}  // namespace slab
