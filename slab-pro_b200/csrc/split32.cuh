// FP32 split-precision step loop: data layout shared by the single-scenario
// path, the batched path and the server.
//
// Particles. A position is an int32 base cell (ib << 16 | jb) plus an FP32
// offset f = x/dx - ib in [0.5, 1.5): the quadratic B-spline stencil of the
// particle is nodes ib..ib+2 (the reference's i_base = int(x/dx - 0.5),
// src/simulation.cpp:741-742). Offsets stay O(1), so km-scale domains keep
// ~1e-7 dx resolution where an absolute FP32 coordinate would keep ~1e-3 m.
// Per particle (SoA): cell 4 B, f 8, v 8, h 4, m 4, id 4; vz and z only in
// steps that feed an output frame.
//
// Sparse tiles. Base cells are grouped in TILE x TILE tiles. Particles are
// stored per tile: G2P writes tile t's particles into t's segment of the
// next buffer, those still in t from the front, those that moved to one of
// the 8 neighbour tiles from the back (double buffered). The next step
// collects a tile's particles from its own stayers and its neighbours'
// movers. Nothing is sorted globally.
//
// Nodes. Node (i, j) is owned by tile (i / TILE, j / TILE). Per-step grid
// fields and the persistent h_max / v_max2 live in TILE x TILE node blocks
// allocated on first touch from a pool. P2G writes, per active tile, partial
// sums over its (TILE+2)^2 node window; the grid update adds the partials of
// the up-to-4 tiles covering a node in a fixed order, so every sum has a
// fixed order and results are bitwise reproducible.
#pragma once

#include "common.cuh"

namespace slab {

#ifndef SLAB_TILE
#define SLAB_TILE 8
#endif
constexpr int TILE = SLAB_TILE;       // base cells per tile edge (8 or 16)
static_assert(TILE == 8 || TILE == 16, "tile edge must be 8 or 16 cells");
constexpr int TN = TILE + 2;          // node window edge of a tile
constexpr int NCELL = TILE * TILE;    // cells per tile = threads per CTA
constexpr int NQ = 7;                 // P2G sums: m, m vx, m vy, m h, Fx, Fy, m vz
constexpr int PART_STRIDE = NQ * TN * TN;  // floats per tile partial
constexpr int CHUNK = 1024;           // particles staged per pass of P2G/G2P
constexpr int PARTICLE_PAD = 16;      // elements allocated past the last particle of every particle array

__host__ __device__ inline int32_t pack_cell(int ib, int jb) { return (ib << 16) | jb; }
__host__ __device__ inline int cell_i(int32_t c) { return (int)((uint32_t)c >> 16); }
__host__ __device__ inline int cell_j(int32_t c) { return (int)(c & 0xffff); }

struct PBuf {
    int32_t* cell;
    float2* f;
    float2* v;
    float* h;
    float* m;
    int32_t* id;
    float* vz;
    float* z;
};

// Per-scenario counters (device).
struct SCnt {
    int32_t act_count[2];  // active tiles of the list of each parity
    int32_t cursor;        // particles placed in the next buffer
    int32_t seq;           // completed G2P passes (buffer parity = seq & 1)
    int32_t stepid;        // P2G passes so far (stamps grid tiles / blocks)
    int32_t vz_next;       // the running G2P must store vz (a frame may follow)
    int32_t outs;          // the running step writes output fields
    double grid_mass;      // FP64 sum of node masses of the last grid update
    int32_t t0_pending;    // the scenario still needs simulate()'s t=0 pass
    int32_t vz_valid;      // buffer vz / z were written by the last G2P (an output step)
};

// Work descriptor of one active tile t for the running step (written by
// k_prep). Its particles are found in 9 candidate ranges of the current
// buffer: range 4 holds the stayers of t's own segment, range d != 4 the
// movers of neighbour t - dir(d) (of which only those now in t are used);
// rpref[d] is the number of candidates before range d; total is the exact
// particle count of t.
struct TileDesc {
    int32_t t, total, nxt_off, sid;
    int32_t rstart[9];
    int32_t rpref[10];
    int32_t blk4[4];  // node blocks of the tile's node window (own, +y, +x, +xy grid tile), written by k_grid
    int32_t pad_;
};

// Segment record of a tile in a particle buffer (GRP_STRIDE ints, one
// 64-byte line): [0] first stayer, [1] first mover (= end of stayers),
// [2] end, [3 + d] number of particles that moved in direction d (d = 4: the
// stayers), [GRP_STAMP] the step (seq) the record belongs to -- a record
// with another stamp is stale.
constexpr int GRP_STRIDE = 16;
constexpr int GRP_STAMP = 12;

// Device descriptor of one scenario.
struct Scn {
    Ctl* ctl;
    SCnt* cnt;
    // physics (FP32 copies of slab_params)
    float g, rho, fr, ood;
    int32_t fric;
    float mu_c, mu_v, xi, mu1, mu2, I0, d, phi;
    int32_t Np;
    PBuf buf[2];
    int32_t* grp[2];        // [ntiles][GRP_STRIDE] segment records (see GRP_STRIDE)
    int32_t* act_stamp;     // [ntiles] last seq the tile was put on an active list
    int32_t* act_list[2];   // active tiles of each parity
    int32_t* slot_of;       // [ntiles] work index (partial slot) of the tile in the running step
    int32_t* nxt_off;       // [ntiles] start of the tile's segment in the next buffer
    int32_t* gt_stamp;      // [ntiles] stepid at which the tile joined the grid list
    int32_t* blk_of;        // [ntiles] node block of the tile, -1 if none yet
    int32_t act_cap;
    int32_t pad_;
};

// Shared by all scenarios of a context: terrain and node-block pool.
struct Shared {
    int32_t Nx, Ny, TX, TY;
    const float4* dem;  // gx, gy, cos(theta), z per node
    // node blocks, NCELL nodes each
    float4* nv;        // vx, vy, flip x, flip y
    float* hmax;       // persistent maxima
    float* vmax2;
    float* oh;         // output fields (frame steps)
    float* om;
    float* ovz;
    float* oFx;        // P2G force sums (Grid::F) of frame steps
    float* oFy;
    int32_t* blk_stamp;   // stepid of the last grid update of the block
    int32_t* blk_owner;   // scenario of the block
    int32_t* blk_count;
    int32_t blk_cap;
    int32_t nscn;
    const Scn* scn;
    SCnt* cnt;            // [nscn] step counters (scn[s].cnt == cnt + s)
    int32_t* work_pref;   // [nscn+1] prefix of active tiles (P2G / G2P work)
    int32_t* wlist;       // [2][work_cap] work items of the two P2G kernels: dense tiles, then sparse ones
    int32_t* wcount;      // [2] their counts
    int32_t split_min;    // tiles with more particles go to the dense kernel; < 0: one P2G kernel for all
    int32_t pad3_;
    int32_t* gflat;       // [gcap][2] grid tiles of the running step: (scenario, grid tile)
    int32_t* gcount;      // entries in gflat
    int32_t gcap;
    int32_t pad2_;
    TileDesc* desc;       // [work_cap] descriptors of the running step
    float* part;          // [work_cap][PART_STRIDE] P2G partial sums
    int32_t work_cap;
    int32_t pad_;
    int32_t* free_blocks; // node blocks released by retired scenarios
    int32_t* free_count;
};

}  // namespace slab
