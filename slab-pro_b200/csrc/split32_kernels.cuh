// Kernels of the FP32 split-precision step loop, shared by the
// single-scenario path and the batched / served paths. One step is
//   k_prep   (grid)    one thread per active tile: its 9 candidate ranges,
//                      its segment in the next buffer, its grid tiles on the
//                      flat grid-tile list
//   k_p2g_cell, k_p2g_sparse (grid)
//                      one CTA per active tile: P2G partial sums, tiles of
//                      more than split_min particles by the cell-sorted
//                      kernel, the others by the sparse-tile kernel
//   k_grid   (grid)    one CTA per grid tile: grid update + friction
//   k_g2p    (grid)    one CTA per active tile: G2P, advection, regrouping
//   k_end    (1 CTA)   per scenario: end of the step, then the next step's
//                      dt / stop rules and work-list prefix (k_arm_begin does
//                      the same at the start of an advance call)
// The CTAs take contiguous runs of a flat list of work items of all
// scenarios, so one launch advances every running scenario by one step, each
// with its own dt and friction law.
//
// Every result is independent of the timing of the threads: the cell-sorted
// P2G sorts a tile's particles by cell in a stable, data-determined order and
// sums in that order; the sparse-tile P2G and the other fixed-point variants
// add integers, exact and associative; the grid update adds the partials of a node's tiles in a
// fixed order; G2P places particles by block prefix sums in candidate order;
// everything else is per particle or a max/min. So a step is bitwise
// reproducible, alone or inside a batch.
#pragma once

#include <type_traits>

#include "split32.cuh"
#include "tma.cuh"

namespace slab {
namespace k32 {

__device__ __forceinline__ int dir_i(int d) { return d / 3 - 1; }
__device__ __forceinline__ int dir_j(int d) { return d % 3 - 1; }

// flat work index -> (scenario, index in that scenario's list)
__device__ __forceinline__ bool find_work(const int32_t* pref, int nscn, int w, int& sid, int& loc) {
    if (w >= pref[nscn]) return false;
    int lo = 0, hi = nscn;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (pref[mid] <= w) lo = mid; else hi = mid;
    }
    sid = lo;
    loc = w - pref[lo];
    return true;
}

// exclusive prefix over one value per thread (any blockDim <= 1024 that is a
// multiple of 32); s_warp needs blockDim/32 + 1 ints
__device__ int block_exclusive_scan(int v, int* s_warp) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int t = lane < nw ? s_warp[lane] : 0;
        const int t0 = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < nw) s_warp[lane] = t - t0;
        if (lane == nw - 1) s_warp[nw] = t;
    }
    __syncthreads();
    const int r = s_warp[warp] + x - v;
    __syncthreads();
    return r;
}

// atomicAdd of `val` to *addr by the lanes in `mask`; lanes with the same
// address are combined into one atomic. Returns the lane's old value.
__device__ int warp_atomic_add(int* addr, int val, unsigned mask) {
    const unsigned peers = __match_any_sync(mask, (unsigned long long)addr);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    int prefix = 0, total = 0;
    for (unsigned m = peers; m; m &= m - 1) {
        const int l = __ffs(m) - 1;
        const int v = __shfl_sync(peers, val, l);
        if (l < lane) prefix += v;
        total += v;
    }
    int base = 0;
    if (lane == leader) base = atomicAdd(addr, total);
    base = __shfl_sync(peers, base, leader);
    return base + prefix;
}

// warp_atomic_add in two halves, so that several atomics are in flight
// before the first result is used: issue (the leader's atomic), then finish
// (the broadcast of its result)
struct WarpAdd {
    unsigned peers;
    int leader, prefix, base;
};
__device__ __forceinline__ WarpAdd warp_add_issue(int* addr, int val, unsigned mask) {
    WarpAdd a;
    a.peers = __match_any_sync(mask, (unsigned long long)addr);
    const int lane = threadIdx.x & 31;
    a.leader = __ffs(a.peers) - 1;
    a.prefix = 0;
    int total = 0;
    for (unsigned m = a.peers; m; m &= m - 1) {
        const int l = __ffs(m) - 1;
        const int v = __shfl_sync(a.peers, val, l);
        if (l < lane) a.prefix += v;
        total += v;
    }
    a.base = 0;
    if (lane == a.leader) a.base = atomicAdd(addr, total);
    return a;
}
__device__ __forceinline__ int warp_add_finish(const WarpAdd& a) { return __shfl_sync(a.peers, a.base, a.leader) + a.prefix; }

// candidate index -> particle index in the current buffer (range d)
__device__ __forceinline__ int cand_to_index(int q, const TileDesc& D, int& d) {
    d = 0;
    while (d < 8 && D.rpref[d + 1] <= q) ++d;
    return D.rstart[d] + (q - D.rpref[d]);
}

constexpr int DESC_WORDS = (int)(sizeof(TileDesc) / 4);

// copy a descriptor to shared memory (threads 0..27)
__device__ __forceinline__ void load_desc(const TileDesc* g, TileDesc* s) {
    if (threadIdx.x < (int)(sizeof(TileDesc) / 4)) reinterpret_cast<int*>(s)[threadIdx.x] = reinterpret_cast<const int*>(g)[threadIdx.x];
}

__device__ __forceinline__ int tile_of_cell(int32_t cell, int TY) { return (cell_i(cell) / TILE) * TY + cell_j(cell) / TILE; }

// ---------------------------------------------------------------- control

// K5 (first half), run by one CTA: per scenario, the stop rules of the
// running advance call and Simulation::updateDt (ctl_begin), then the
// prefix of active tiles over scenarios (the work list of the step).
// t0_pass: simulate()'s t=0 pass for scenarios that still need it.
__device__ void begin_scenarios(const Shared& sh, int t0_pass) {
    __shared__ int s_warp[33];
    __shared__ int s_tot;
    const int tid = threadIdx.x;
    int total = 0;
    for (int base = 0; base < sh.nscn; base += blockDim.x) {
        const int s = base + tid;
        int cnt = 0;
        if (s < sh.nscn) {
            const Scn& S = sh.scn[s];
            Ctl* c = S.ctl;
            SCnt* n = S.cnt;
            if (t0_pass) {
                if (n->t0_pending) {
                    ctl_begin_t0(c, sh.Nx, sh.Ny);
                    n->t0_pending = 0;
                } else {
                    c->active = 0;
                }
            } else if (n->t0_pending) {
                c->active = 0;  // added after the last t=0 pass: waits for the next one
            } else {
                ctl_begin(c, sh.Nx, sh.Ny);
            }
            if (c->active) {
                n->stepid += 1;
                n->act_count[(n->seq + 1) & 1] = 0;
                n->cursor = 0;
                n->grid_mass = 0.0;
                n->outs = c->write_outputs;
                const int frame_after = c->frame + (c->frame_end ? 1 : 0);
                const double nft = __dmul_rn(c->output_dt, (double)(frame_after + 1));
                n->vz_next = (c->keep_outputs || __dadd_rn(c->new_time, c->dt_max) > nft - 1e-12) ? 1 : 0;
                cnt = n->act_count[n->seq & 1];
            }
        }
        const int ex = block_exclusive_scan(cnt, s_warp);
        if (s < sh.nscn) sh.work_pref[s] = total + ex;
        if (tid == blockDim.x - 1) s_tot = ex + cnt;
        __syncthreads();
        total += s_tot;
        __syncthreads();
    }
    if (tid == 0) {
        sh.work_pref[sh.nscn] = min(total, sh.work_cap);
        if (total > sh.work_cap) atomicOr(&sh.scn[0].ctl->err, ERR_CAPACITY);
        *sh.gcount = 0;
        sh.wcount[0] = 0;
        sh.wcount[1] = 0;
    }
}

__global__ void k_begin(Shared sh, int t0_pass) { begin_scenarios(sh, t0_pass); }

// Start of an advance call: every scenario gets the step budget and the
// frame-stop rule, then the first step begins.
__global__ void k_arm_begin(Shared sh, int64_t steps_left, int stop_at_frame) {
    for (int s = threadIdx.x; s < sh.nscn; s += blockDim.x) {
        Ctl* c = sh.scn[s].ctl;
        c->stop = 0;
        c->frame_hit = 0;
        c->steps_left = steps_left;
        c->stop_at_frame = stop_at_frame;
    }
    __syncthreads();
    begin_scenarios(sh, 0);
}


// The work items of one CTA: a contiguous range of the flat work list, so
// that consecutive items mostly belong to the same scenario.
__device__ __forceinline__ void work_range(int nwork, int& w0, int& w1) {
    const int per = (nwork + (int)gridDim.x - 1) / (int)gridDim.x;
    w0 = min((int)blockIdx.x * per, nwork);
    w1 = min(w0 + per, nwork);
}

// Scenario of the last work item looked up, with the step fields that do not
// change during a launch (so a new item of the same scenario costs no loads).
struct WorkCache {
    int sid = -1, lo = 0, hi = 0, seq = 0, stepid = 0;
};

// Work items of a P2G kernel: class 0 (dense tiles), 1 (sparse tiles), or
// -1 (every active tile, when the step runs one P2G kernel).
__device__ __forceinline__ int p2g_count(const Shared& sh, int cls) {
    return cls < 0 ? sh.work_pref[sh.nscn] : min(sh.wcount[cls], sh.work_cap);
}
__device__ __forceinline__ int p2g_item(const Shared& sh, int cls, int i) { return cls < 0 ? i : sh.wlist[cls * sh.work_cap + i]; }

// K1 (bookkeeping half): a tile's particles are the stayers of its own
// segment in the current buffer plus the movers of the 8 neighbour segments
// that moved to it (those are filtered by cell when read). The descriptor
// records these 9 candidate ranges and the exact count, reserves the tile's
// segment in the next buffer, and puts the 4 tiles owning its node window on
// the grid-tile list.
// Sixteen lanes (half a warp) per active tile, so that its independent
// global accesses go out together: lanes 0-8 read the 9 segment records,
// lanes 9-12 stamp the 4 grid tiles, lane 0 takes the segment cursor and the
// class-list slot; the counts and range prefixes are half-warp shuffles, and
// the lanes write the descriptor's words side by side.
constexpr int PREP_LANES = 16;
constexpr int PREP_THREADS = 256;
static_assert(sizeof(TileDesc) == 28 * 4 && offsetof(TileDesc, rstart) == 4 * 4 && offsetof(TileDesc, rpref) == 13 * 4 &&
                  offsetof(TileDesc, blk4) == 23 * 4,
              "k_prep writes the descriptor word by word");

__device__ __forceinline__ void prep_body(const Shared& sh) {
    const int nwork = sh.work_pref[sh.nscn];
    const int lane = threadIdx.x & 31, r = lane & (PREP_LANES - 1);
    const int per_block = (int)blockDim.x / PREP_LANES;
    const int stride = gridDim.x * per_block;
    // whole warps run every iteration (the shuffles need both halves); a half
    // without a tile computes with valid = false
    for (int w0 = blockIdx.x * per_block; w0 + (int)(threadIdx.x & ~31u) / PREP_LANES < nwork; w0 += stride) {
        const int w = w0 + threadIdx.x / PREP_LANES;
        const bool valid = w < nwork;
        int sid = 0, loc = 0;
        if (valid) find_work(sh.work_pref, sh.nscn, w, sid, loc);
        const Scn& S = sh.scn[sid];
        SCnt* n = sh.cnt + sid;  // no load of S.cnt in the chain
        int seq = 0, stamp = 0, t = 0;
        if (valid) {
            seq = n->seq;
            stamp = n->stepid;
            t = S.act_list[seq & 1][loc];
        }
        const int cur = seq & 1;
        const int ti = t / sh.TY, tj = t % sh.TY;
        // lanes 0-8: the record of neighbour d = r (its particles that moved to t)
        int rs = 0, rl = 0, c = 0;
        if (valid && r < 9) {
            const int si = ti - dir_i(r), sj = tj - dir_j(r);
            if (si >= 0 && sj >= 0 && si < sh.TX && sj < sh.TY) {
                const int32_t* G = S.grp[cur] + (size_t)(si * sh.TY + sj) * GRP_STRIDE;
                if (G[GRP_STAMP] == seq) {
                    const int g0 = G[0], g1 = G[1], g2 = G[2];
                    rs = r == 4 ? g0 : g1;
                    rl = r == 4 ? g1 - g0 : g2 - g1;
                    c = G[3 + r];
                }
            }
        }
        // lanes 9-12: the grid tiles of t's node window, stamped with this step
        bool new_gt = false;
        int gt = 0;
        if (valid && r >= 9 && r < 13) {
            const int k = r - 9;
            const int gi = ti + (k >> 1), gj = tj + (k & 1);
            if (gi < sh.TX && gj < sh.TY) {
                gt = gi * sh.TY + gj;
                new_gt = atomicMax(&S.gt_stamp[gt], stamp) < stamp;
            }
        }
        // half-warp shuffles: the tile's particle count and the range prefixes
        int incl = rl;
#pragma unroll
        for (int o = 1; o < PREP_LANES; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o, PREP_LANES);
            if (r >= o) incl += y;
        }
        int cnt = c;
#pragma unroll
        for (int o = PREP_LANES / 2; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o, PREP_LANES);
        const int ncand = __shfl_sync(0xffffffffu, incl, 8, PREP_LANES);
        // lane 0: the segment cursor and the class list (one atomic per address and warp)
        const bool leader = valid && r == 0;
        const unsigned lmask = __ballot_sync(0xffffffffu, leader);
        int nxt_off = 0;
        if (leader) {
            const WarpAdd a_cur = warp_add_issue(&n->cursor, cnt, lmask);
            const int cls = cnt > sh.split_min ? 0 : 1;
            WarpAdd a_cls{};
            if (sh.split_min >= 0) a_cls = warp_add_issue(sh.wcount + cls, 1, lmask);
            nxt_off = warp_add_finish(a_cur);
            if (sh.split_min >= 0) {  // dense tiles to the cell-sorted P2G, sparse ones to the fixed-point P2G
                const int at = warp_add_finish(a_cls);
                if (at < sh.work_cap) sh.wlist[cls * sh.work_cap + at] = w;
            }
            S.slot_of[t] = w;
        }
        // the new grid tiles onto the flat grid-tile list, in lane order
        const unsigned gmask = __ballot_sync(0xffffffffu, new_gt);
        const unsigned hbits = (lane < PREP_LANES ? 0x0000ffffu : 0xffff0000u);
        const int ng = __popc(gmask & hbits);
        int at_g = 0;
        if (leader) at_g = warp_atomic_add(sh.gcount, ng, lmask);
        at_g = __shfl_sync(0xffffffffu, at_g, lane & ~(PREP_LANES - 1));
        nxt_off = __shfl_sync(0xffffffffu, nxt_off, lane & ~(PREP_LANES - 1));
        if (new_gt) {
            const int at = at_g + __popc(gmask & hbits & ((1u << lane) - 1u));
            if (at < sh.gcap) {
                sh.gflat[2 * at] = sid;
                sh.gflat[2 * at + 1] = gt;
            } else {
                atomicOr(&S.ctl->err, ERR_CAPACITY);
            }
        }
        // the descriptor, word by word (TileDesc: t, total, nxt_off, sid,
        // rstart[9], rpref[10], blk4[4], pad)
        if (valid) {
            int* D = reinterpret_cast<int*>(sh.desc + w);
            if (r < 9) {
                D[4 + r] = rs;
                D[13 + r] = incl - rl;  // candidates before range r
            } else if (r == 9) {
                D[22] = ncand;
            } else if (r < 14) {
                D[23 + (r - 10)] = -1;  // grid tiles off the terrain keep -1; k_grid fills the others
            } else if (r == 14) {
                D[27] = 0;
            } else {
                D[0] = t;
                D[1] = cnt;
                D[2] = nxt_off;
                D[3] = sid;
            }
        }
    }
}

__global__ void __launch_bounds__(PREP_THREADS) k_prep(Shared sh) { prep_body(sh); }

// ------------------------------------------------------------------- P2G

constexpr int P2G_THREADS = NCELL;  // one thread per cell slot; the CTA strides over its tile's particles
constexpr int P2G_MIN_BLOCKS = NCELL == 64 ? 16 : 4;

// Fixed-point accumulation schemes of k_p2g:
//  ACC_I32   one int32 per sum, 2^-30 of the tile's bound
//  ACC_HILO  int32 pair: the rounded contribution and, 2^-20 finer, the
//            part below one quantum -- each contribution keeps about FP32
//            precision relative to itself; two plain (non-returning) atomics
//  ACC_I64   one int64 per sum at 2^-52 of the bound
//  ACC_CELL  no fixed point: k_p2g_cell, FP32 sums over cell-sorted particles
//  ACC_WARP  k_p2g_warp: ACC_HILO sums with one warp per tile
//  ACC_MIXED dense tiles (more than split_min particles) by k_p2g_cell, the
//            others by k_p2g_sparse (64-bit fixed point): each tile's scheme
//            depends only on its particle count, so results are still
//            reproducible
enum { ACC_I32 = 0, ACC_HILO = 1, ACC_I64 = 2, ACC_CELL = 3, ACC_WARP = 4, ACC_MIXED = 5 };

struct P2GSmem {
    long long node[NQ * TN * TN];  // fixed-point sums of the (TILE+2)^2 window (int32 pairs / int64)
    float4 dem[(TILE + 1) * (TILE + 1)];
    int ccnt[NCELL];
    unsigned bmax[NQ];             // per-quantity bound of one contribution (float bits)
    int mcc;                       // most particles in one cell of the tile
    float scale[NQ], iscale[NQ];
    TileDesc d;
};

// Per-particle P2G quantities (src/simulation.cpp:729-756): mass, momentum,
// m vz, m h, and for the force K = m g cos^2(theta) with the slope of the
// containing cell (src/complex_terrain.cpp:113-130) and the depth-averaged
// pressure sigma = -rho g cos^2 h / 2 with h A = m / rho.
struct PQ {
    float fx, fy, m, mvx, mvy, mh, mvz, Kgx, Kgy, Khh;
    int li, lj;
};

__device__ __forceinline__ PQ load_pq(const PBuf& B, int src, int li, int lj, const float4* dem, float g, float hod, bool outs) {
    PQ p;
    const float2 f = B.f[src], v = B.v[src];
    const float h = B.h[src], m = B.m[src];
    const float4 dm = dem[(li + (f.x >= 1.f ? 1 : 0)) * (TILE + 1) + (lj + (f.y >= 1.f ? 1 : 0))];
    const float K = m * g * dm.z * dm.z;
    p.fx = f.x;
    p.fy = f.y;
    p.m = m;
    p.mvx = m * v.x;
    p.mvy = m * v.y;
    p.mh = m * h;
    p.mvz = outs ? m * B.vz[src] : 0.f;
    p.Kgx = K * dm.x;
    p.Kgy = K * dm.y;
    p.Khh = K * h * hod;
    p.li = li;
    p.lj = lj;
    return p;
}

// K2: P2G of one tile (src/simulation.cpp:726-798), one thread per particle,
// sums in 32-bit fixed point with shared-memory integer atomics. Integer
// addition is exact and associative, so the sums do not depend on the order
// in which particles arrive: the result is bitwise reproducible without
// sorting. Pass A finds, per quantity, a bound b on one contribution and the
// largest particle count of a cell; a node's sum then stays below
// 9 * cells_max * 0.75 * b, and the scale 2^e is the largest power of two
// that keeps that below 2^30. The resolution is 2^-30 of that bound, finer
// than FP32 relative to the largest contribution. Pass B adds the
// contributions; the window is converted back and written as the partials.
template <int ACC>
__global__ void __launch_bounds__(P2G_THREADS, P2G_MIN_BLOCKS) k_p2g(Shared sh, int cls) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    P2GSmem& sm = *reinterpret_cast<P2GSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31;
    int i0, i1;
    work_range(p2g_count(sh, cls), i0, i1);
    for (int i = i0; i < i1; ++i) {
        const int w = p2g_item(sh, cls, i);
        load_desc(sh.desc + w, &sm.d);
        for (int k = tid; k < NQ * TN * TN; k += P2G_THREADS) sm.node[k] = 0;
        int* node32 = reinterpret_cast<int*>(sm.node);  // ACC_I32: [q][node]; ACC_HILO: hi at [q][node], lo at NQ*TN*TN + [q][node]
        for (int k = tid; k < NCELL; k += P2G_THREADS) sm.ccnt[k] = 0;
        if (tid < NQ) sm.bmax[tid] = 0u;
        if (tid == 0) sm.mcc = 0;
        __syncthreads();
        const Scn& S = sh.scn[sm.d.sid];
        const int t = sm.d.t;
        const int ti = t / sh.TY, tj = t % sh.TY;
        SCnt* n = S.cnt;
        const int cur = n->seq & 1;
        const bool outs = n->outs != 0;
        for (int k = tid; k < (TILE + 1) * (TILE + 1); k += P2G_THREADS) {
            const int i = ti * TILE + k / (TILE + 1), j = tj * TILE + k % (TILE + 1);
            sm.dem[k] = (i < sh.Nx && j < sh.Ny) ? sh.dem[(int64_t)i * sh.Ny + j] : make_float4(0.f, 0.f, 1.f, 0.f);
        }
        __syncthreads();
        const int ncand = sm.d.rpref[9];
        const PBuf B = S.buf[cur];
        const float g = S.g, hod = 0.5f * S.ood;
        // pass A: bounds and cell counts
        float bm = 0.f, bvx = 0.f, bvy = 0.f, bh = 0.f, bvz = 0.f, bF = 0.f;
        for (int k = tid; k < ncand; k += P2G_THREADS) {
            int d;
            const int src = cand_to_index(k, sm.d, d);
            const int32_t cell = B.cell[src];
            const int li = cell_i(cell) - ti * TILE, lj = cell_j(cell) - tj * TILE;
            if ((unsigned)li >= TILE || (unsigned)lj >= TILE) {
                if (d == 4) atomicOr(&S.ctl->err, ERR_MOVE);  // a stayer outside its tile
                continue;
            }
            const PQ p = load_pq(B, src, li, lj, sm.dem, g, hod, outs);
            const int c = atomicAdd(&sm.ccnt[li * TILE + lj], 1) + 1;
            atomicMax(&sm.mcc, c);
            bm = fmaxf(bm, p.m);
            bvx = fmaxf(bvx, fabsf(p.mvx));
            bvy = fmaxf(bvy, fabsf(p.mvy));
            bh = fmaxf(bh, p.mh);
            bvz = fmaxf(bvz, fabsf(p.mvz));
            bF = fmaxf(bF, p.Khh + fmaxf(fabsf(p.Kgx), fabsf(p.Kgy)));
        }
        bm = warp_max(bm);
        bvx = warp_max(bvx);
        bvy = warp_max(bvy);
        bh = warp_max(bh);
        bvz = warp_max(bvz);
        bF = warp_max(bF);
        if (lane == 0) {
            atomicMax(&sm.bmax[0], __float_as_uint(bm));
            atomicMax(&sm.bmax[1], __float_as_uint(bvx));
            atomicMax(&sm.bmax[2], __float_as_uint(bvy));
            atomicMax(&sm.bmax[3], __float_as_uint(bh));
            atomicMax(&sm.bmax[4], __float_as_uint(bF));
            atomicMax(&sm.bmax[5], __float_as_uint(bF));
            atomicMax(&sm.bmax[6], __float_as_uint(bvz));
        }
        __syncthreads();
        if (tid < NQ) {
            const float bound = 9.f * (float)sm.mcc * 0.75f * __uint_as_float(sm.bmax[tid]);
            int e = 0;
            if (bound > 0.f) {
                int E;
                frexpf(bound, &E);  // bound < 2^E
                e = min(max((ACC == ACC_I64 ? 52 : 30) - E, -120), 120);
            }
            sm.scale[tid] = ldexpf(1.f, e);
            sm.iscale[tid] = ldexpf(1.f, -e);
        }
        __syncthreads();
        const float s0 = sm.scale[0], s1 = sm.scale[1], s2 = sm.scale[2], s3 = sm.scale[3], s4 = sm.scale[4], s5 = sm.scale[5],
                    s6 = sm.scale[6];
        const int lob = lo_bits_for(9 * sm.mcc);  // lo sums of a node stay below 2^30
        const float lo_mul = ldexpf(1.f, lob);
        const double lo_div = ldexp(1.0, -lob);
        // pass B: fixed-point contributions
        for (int k = tid; k < ncand; k += P2G_THREADS) {
            int d;
            const int src = cand_to_index(k, sm.d, d);
            const int32_t cell = B.cell[src];
            const int li = cell_i(cell) - ti * TILE, lj = cell_j(cell) - tj * TILE;
            if ((unsigned)li >= TILE || (unsigned)lj >= TILE) continue;
            const PQ p = load_pq(B, src, li, lj, sm.dem, g, hod, outs);
            float wx[3], wy[3], dwx[3], dwy[3];
            bspline3(p.fx, wx, dwx);
            bspline3(p.fy, wy, dwy);
#pragma unroll
            for (int a = 0; a < 3; ++a) {
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    const float wgt = wx[a] * wy[b];
                    if (wgt > 3e-3f) {  // the reference's weight cut-off (src/simulation.cpp:780)
                        const int nd = (li + a) * TN + (lj + b);
                        const float c[NQ] = {p.m * wgt, p.mvx * wgt, p.mvy * wgt, p.mh * wgt, p.Khh * (dwx[a] * wy[b]) - p.Kgx * wgt,
                                             p.Khh * (dwy[b] * wx[a]) - p.Kgy * wgt, p.mvz * wgt};
                        const float sc[NQ] = {s0, s1, s2, s3, s4, s5, s6};
#pragma unroll
                        for (int q = 0; q < NQ; ++q) {
                            if (q == 6 && !outs) continue;
                            if (ACC == ACC_I64) {
                                atomicAdd(reinterpret_cast<unsigned long long*>(sm.node + q * TN * TN + nd),
                                          (unsigned long long)__float2ll_rn(c[q] * sc[q]));
                            } else {
                                const float x = c[q] * sc[q];
                                const int hi = __float2int_rn(x);
                                atomicAdd(node32 + q * TN * TN + nd, hi);
                                if (ACC == ACC_HILO) {
                                    const int lo = __float2int_rn((x - (float)hi) * lo_mul);
                                    if (lo) atomicAdd(node32 + (NQ + q) * TN * TN + nd, lo);
                                }
                            }
                        }
                    }
                }
            }
        }
        __syncthreads();
        float* P = sh.part + (size_t)w * PART_STRIDE;
        for (int k = tid; k < PART_STRIDE; k += P2G_THREADS) {
            const float is = sm.iscale[k / (TN * TN)];
            float v;
            if (ACC == ACC_I64) v = (float)((double)sm.node[k] * (double)is);
            else if (ACC == ACC_HILO) v = (float)(((double)node32[k] + (double)node32[NQ * TN * TN + k] * lo_div) * (double)is);
            else v = (float)node32[k] * is;
            P[k] = v;
        }
        __syncthreads();
    }
}

// --------------------------------------- P2G, one warp per tile (fixed point)

constexpr int P2W_WARPS = TILE == 8 ? 8 : 2;  // tiles in flight per CTA
constexpr int P2W_THREADS = 32 * P2W_WARPS;
constexpr int P2W_REG = 1;                     // chunks of 32 candidates a lane keeps between the passes

struct P2WWarp {
    int node[2 * NQ * TN * TN];  // fixed-point sums of the tile's node window: hi [q][node], then lo
    int ccnt[NCELL];             // particles per cell
    TileDesc d;
};

// P2G quantities of one candidate of tile (ti, tj), with the slope of its
// containing cell read from the FP32 terrain copy; valid = in the tile
__device__ __forceinline__ PQ warp_pq(const Shared& sh, const PBuf& B, const TileDesc& D, int k, int ti, int tj, float g, float hod, bool outs,
                                      bool& valid, bool& stayer) {
    int d;
    const int src = cand_to_index(k, D, d);
    const int32_t cell = B.cell[src];
    const float2 f = B.f[src], v = B.v[src];
    const float h = B.h[src], m = B.m[src];
    const float vz = outs ? B.vz[src] : 0.f;
    const int ci = cell_i(cell), cj = cell_j(cell);
    const int li = ci - ti * TILE, lj = cj - tj * TILE;
    valid = (unsigned)li < TILE && (unsigned)lj < TILE;
    stayer = d == 4;
    PQ p;
    p.li = li;
    p.lj = lj;
    p.fx = f.x;
    p.fy = f.y;
    if (!valid) {
        p.m = p.mvx = p.mvy = p.mh = p.mvz = p.Kgx = p.Kgy = p.Khh = 0.f;
        return p;
    }
    const float4 dm = sh.dem[(int64_t)(ci + (f.x >= 1.f ? 1 : 0)) * sh.Ny + (cj + (f.y >= 1.f ? 1 : 0))];
    const float K = m * g * dm.z * dm.z;
    p.m = m;
    p.mvx = m * v.x;
    p.mvy = m * v.y;
    p.mh = m * h;
    p.mvz = m * vz;
    p.Kgx = K * dm.x;
    p.Kgy = K * dm.y;
    p.Khh = K * h * hod;
    return p;
}

// K2 variant: P2G of one tile (src/simulation.cpp:726-798) by one warp, so
// that many tiles are in flight on an SM with no block-wide barrier. The
// sums are 32-bit fixed-point pairs in the warp's shared-memory node window,
// added with integer atomics: exact and associative, so the result does not
// depend on the order of the particles (bitwise reproducible, the same alone
// or inside a batch). Pass A bounds one contribution per quantity (b) and the
// particles of one cell (mcc); a node's sum stays below 9 * mcc * 0.75 * b,
// and the scale is the largest power of two that keeps that below 2^30; the
// hi word is the rounded contribution, the lo word the rest at 2^-20.
__global__ void __launch_bounds__(P2W_THREADS, 3) k_p2g_warp(Shared sh, int cls) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    P2WWarp& sw = reinterpret_cast<P2WWarp*>(smem_raw)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * P2W_WARPS + (threadIdx.x >> 5), nw = gridDim.x * P2W_WARPS;
    const int nwork = p2g_count(sh, cls);
    const int per = (nwork + nw - 1) / nw;
    const int i0 = min(gw * per, nwork), i1 = min(i0 + per, nwork);
    int* hi = sw.node;
    int* lo = sw.node + NQ * TN * TN;
    for (int i = i0; i < i1; ++i) {
        const int w = p2g_item(sh, cls, i);
        if (lane < (int)(sizeof(TileDesc) / 4)) reinterpret_cast<int*>(&sw.d)[lane] = reinterpret_cast<const int*>(sh.desc + w)[lane];
        for (int k = lane; k < 2 * NQ * TN * TN; k += 32) sw.node[k] = 0;
        for (int k = lane; k < NCELL; k += 32) sw.ccnt[k] = 0;
        __syncwarp();
        const TileDesc& D = sw.d;
        const Scn& S = sh.scn[D.sid];
        const SCnt* n = S.cnt;
        const int cur = n->seq & 1;
        const bool outs = n->outs != 0;
        const int ti = D.t / sh.TY, tj = D.t % sh.TY;
        const int ncand = D.rpref[9];
        const PBuf B = S.buf[cur];
        const float g = S.g, hod = 0.5f * S.ood;
        // pass A: bounds and cell counts (the first chunks stay in registers)
        PQ keep[P2W_REG];
        bool kval[P2W_REG];
        float bm = 0.f, bvx = 0.f, bvy = 0.f, bh = 0.f, bvz = 0.f, bF = 0.f;
        int mcc = 0;
        for (int c = 0, k0 = 0; k0 < ncand; ++c, k0 += 32) {
            const int k = k0 + lane;
            bool valid = false, stayer = false;
            PQ p;
            if (k < ncand) p = warp_pq(sh, B, D, k, ti, tj, g, hod, outs, valid, stayer);
            if (k < ncand && !valid && stayer) atomicOr(&S.ctl->err, ERR_MOVE);  // a stayer outside its tile
#pragma unroll
            for (int r = 0; r < P2W_REG; ++r)
                if (c == r) {
                    keep[r] = p;
                    kval[r] = valid;
                }
            if (valid) {
                mcc = max(mcc, atomicAdd(&sw.ccnt[p.li * TILE + p.lj], 1) + 1);
                bm = fmaxf(bm, p.m);
                bvx = fmaxf(bvx, fabsf(p.mvx));
                bvy = fmaxf(bvy, fabsf(p.mvy));
                bh = fmaxf(bh, p.mh);
                bvz = fmaxf(bvz, fabsf(p.mvz));
                bF = fmaxf(bF, p.Khh + fmaxf(fabsf(p.Kgx), fabsf(p.Kgy)));
            }
        }
        bm = warp_max(bm);
        bvx = warp_max(bvx);
        bvy = warp_max(bvy);
        bh = warp_max(bh);
        bvz = warp_max(bvz);
        bF = warp_max(bF);
        for (int o = 16; o > 0; o >>= 1) mcc = max(mcc, __shfl_xor_sync(0xffffffffu, mcc, o));
        const float bq[NQ] = {bm, bvx, bvy, bh, bF, bF, bvz};
        float sc[NQ], isc[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            const float bound = 9.f * (float)mcc * 0.75f * bq[q];
            int e = 0;
            if (bound > 0.f) {
                int E;
                frexpf(bound, &E);  // bound < 2^E
                e = min(max(30 - E, -120), 120);
            }
            sc[q] = ldexpf(1.f, e);
            isc[q] = ldexpf(1.f, -e);
        }
        const int lob = lo_bits_for(9 * mcc);  // lo sums of a node stay below 2^30
        const float lo_mul = ldexpf(1.f, lob);
        const double lo_div = ldexp(1.0, -lob);
        // pass B: fixed-point contributions
        for (int c = 0, k0 = 0; k0 < ncand; ++c, k0 += 32) {
            const int k = k0 + lane;
            bool valid = false, stayer = false;
            PQ p;
            if (c < P2W_REG) {
#pragma unroll
                for (int r = 0; r < P2W_REG; ++r)
                    if (c == r) {
                        p = keep[r];
                        valid = kval[r];
                    }
            } else if (k < ncand) {
                p = warp_pq(sh, B, D, k, ti, tj, g, hod, outs, valid, stayer);
            }
            if (!valid) continue;
            float wx[3], wy[3], dwx[3], dwy[3];
            bspline3(p.fx, wx, dwx);
            bspline3(p.fy, wy, dwy);
#pragma unroll
            for (int a = 0; a < 3; ++a) {
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    const float wgt = wx[a] * wy[b];
                    if (wgt > 3e-3f) {  // the reference's weight cut-off (src/simulation.cpp:780)
                        const int nd = (p.li + a) * TN + (p.lj + b);
                        const float cq[NQ] = {p.m * wgt, p.mvx * wgt, p.mvy * wgt, p.mh * wgt, p.Khh * (dwx[a] * wy[b]) - p.Kgx * wgt,
                                              p.Khh * (dwy[b] * wx[a]) - p.Kgy * wgt, p.mvz * wgt};
#pragma unroll
                        for (int q = 0; q < NQ; ++q) {
                            if (q == 6 && !outs) continue;
                            const float x = cq[q] * sc[q];
                            const int h_ = __float2int_rn(x);
                            atomicAdd(hi + q * TN * TN + nd, h_);
                            const int l_ = __float2int_rn((x - (float)h_) * lo_mul);
                            if (l_) atomicAdd(lo + q * TN * TN + nd, l_);
                        }
                    }
                }
            }
        }
        __syncwarp();
        float* P = sh.part + (size_t)w * PART_STRIDE;
        for (int k = lane; k < PART_STRIDE; k += 32) {
            const int q = k / (TN * TN);
            float is = isc[0];
#pragma unroll
            for (int r = 1; r < NQ; ++r)
                if (q == r) is = isc[r];
            P[k] = (float)(((double)hi[k] + (double)lo[k] * lo_div) * (double)is);
        }
        __syncwarp();
    }
}

// ------------------------------------------------ P2G over cell-sorted particles

// Optional per-phase cycle counters of the P2G kernel (builds with
// -DSLAB_PHASE_CLOCKS only): thread 0 of each CTA adds the clock64 cycles of
// each phase of each tile to g_phase_clk[phase] (cell P2G 0-6, G2P 8-12);
// g_phase_clk[15] and [14] count their tiles.
#ifdef SLAB_PHASE_CLOCKS
__device__ unsigned long long g_phase_clk[16];
#define SLAB_PHASE_BEGIN long long t_prev_ = clock64()
#define SLAB_PHASE_MARK(k)                                                  \
    do {                                                                    \
        if (threadIdx.x == 0) {                                             \
            const long long c_ = clock64();                                 \
            atomicAdd(&g_phase_clk[k], (unsigned long long)(c_ - t_prev_)); \
            t_prev_ = c_;                                                   \
        }                                                                   \
    } while (0)
#define SLAB_PHASE_TILE()                                         \
    do {                                                          \
        if (threadIdx.x == 0) atomicAdd(&g_phase_clk[15], 1ull); \
    } while (0)
#define SLAB_PHASE_TILE_G2P()                                     \
    do {                                                          \
        if (threadIdx.x == 0) atomicAdd(&g_phase_clk[14], 1ull); \
    } while (0)
#else
#define SLAB_PHASE_BEGIN
#define SLAB_PHASE_MARK(k)
#define SLAB_PHASE_TILE()
#define SLAB_PHASE_TILE_G2P()
#endif

// index of work item w in its scenario's list (pref: the prefix over scenarios)
__device__ __forceinline__ int cached_work(const Shared& sh, const int32_t* pref, int w, WorkCache& c) {
    if (w < c.lo || w >= c.hi) {
        int loc;
        find_work(pref, sh.nscn, w, c.sid, loc);
        c.lo = pref[c.sid];
        c.hi = pref[c.sid + 1];
        const SCnt* n = sh.scn[c.sid].cnt;
        c.seq = n->seq;
        c.stepid = n->stepid;
    }
    return w - c.lo;
}


constexpr int P2C_THREADS = NCELL;  // one thread per cell of the tile
#ifndef SLAB_P2C_MIN_BLOCKS
#define SLAB_P2C_MIN_BLOCKS (NCELL == 64 ? 12 : 3)
#endif
constexpr int P2C_MIN_BLOCKS = SLAB_P2C_MIN_BLOCKS;  // resident CTAs per SM the register budget is cut for
constexpr int P2C_WARPS = P2C_THREADS / 32;
constexpr int NSLOT = 9;            // nodes a cell's particles reach (3 x 3)
constexpr int P2C_CAP = 6 * NCELL;  // candidates of a tile staged in shared memory (more go through global memory)

struct P2CStage {
    float4 sa[P2C_CAP];  // staged candidates, by candidate index: f.x, f.y, m, h
    float2 sv[P2C_CAP];  //                                        v
    float svz[P2C_CAP];  //                                        vz
};

struct P2CSmem {
    P2CStage st;
    float nsum[NQ * TN * TN];  // node sums of the tile's window, [q][node]
    int16_t lc[P2C_CAP];   // local cell of each staged candidate (-1: not in the tile)
    union {
        int32_t ccell[P2C_CAP];  // phase 1: cell of each staged candidate
        int16_t idx[P2C_CAP];    // phases 3-4: sorted position -> candidate index
    };
    alignas(128) float4 dem[(TILE + 1) * (TILE + 1)];  // a tensor copy's destination: 128-byte aligned
    alignas(8) uint64_t dem_bar;  // completion of the terrain window's tensor copy (k_p2g_cell<false>)
    int wcur[P2C_WARPS][NCELL];  // per-warp cell counts, then per-warp write cursors
    int s_warp[33];
    TileDesc d;
    // the scenario of the CTA's current run of tiles (loaded when it changes)
    PBuf B;             // current particle buffer
    int32_t* nxt_cell;  // cell array of the next buffer (sorted index lists of large tiles)
    Ctl* ctl;
    float g, hod;
    int csid, outs;
};

// Bulk-copy staging of the next tile (k_p2g_cell<true>): its 9 candidate
// ranges of the particle arrays, each rounded out to 16-byte boundaries, and
// its terrain window, copied by the TMA engine while the current tile is
// summed. 4-byte arrays take at most 6 extra elements per range, 8-byte ones 2.
constexpr int P2C_SCAP4 = (P2C_CAP + 9 * 6 + 3) / 4 * 4;
constexpr int P2C_SCAP8 = (P2C_CAP + 9 * 2 + 1) / 2 * 2;
constexpr int DEM_W = TILE + 1;  // terrain window edge (nodes)

struct alignas(16) P2CTmaStage {
    int32_t cell[P2C_SCAP4];
    float h[P2C_SCAP4];
    float m[P2C_SCAP4];
    float vz[P2C_SCAP4];
    float2 f[P2C_SCAP8];
    float2 v[P2C_SCAP8];
};
static_assert(P2C_SCAP4 * 4 % 16 == 0 && P2C_SCAP8 * 8 % 16 == 0, "16-byte aligned stage arrays");

struct P2CSmemTma : P2CSmem {
    P2CTmaStage ts;                             // the tile's candidates (until its phase 1 has read them)
    alignas(16) float4 dem2[2][DEM_W * DEM_W];  // terrain windows of this and the next tile
    alignas(8) uint64_t bar;                    // completion of the staged copies
    TileDesc dnext;                             // the next tile's descriptor
    int lead4[9], lead8[9];                     // stage index of each range's first candidate (4-byte / 8-byte arrays)
    int use_stage, dem_staged[2];               // the tile's candidates / terrain windows came by bulk copy
};

// Thread 0: lays out the 9 ranges of tile D in the stage and starts their
// bulk copies (and the terrain window's rows into dem2[slot]) on sm.bar.
// Candidates that do not fit leave the tile to the load path (use_stage 0).
// The particle arrays are padded past Np, so a range rounded up to 16 bytes
// stays inside its allocation.
__device__ __forceinline__ void p2c_issue_stage(P2CSmemTma& sm, const TileDesc& D, const PBuf& B, bool outs, const Shared& sh, int slot) {
    int o4 = 0, o8 = 0;
    bool fit = D.rpref[9] <= P2C_CAP;
    int a4[9], n4[9], a8[9], n8[9];
#pragma unroll
    for (int d = 0; d < 9; ++d) {
        const int rs = D.rstart[d], rl = D.rpref[d + 1] - D.rpref[d];
        a4[d] = rs & ~3;
        n4[d] = rl > 0 ? ((rs + rl + 3) & ~3) - a4[d] : 0;
        a8[d] = rs & ~1;
        n8[d] = rl > 0 ? ((rs + rl + 1) & ~1) - a8[d] : 0;
        sm.lead4[d] = o4 + (rs - a4[d]);
        sm.lead8[d] = o8 + (rs - a8[d]);
        o4 += n4[d];
        o8 += n8[d];
    }
    if (o4 > P2C_SCAP4 || o8 > P2C_SCAP8) fit = false;
    // the terrain window by rows when it lies inside the terrain
    const int ti = D.t / sh.TY, tj = D.t % sh.TY;
    const bool dem_in = ti * TILE + TILE < sh.Nx && tj * TILE + TILE < sh.Ny;
    sm.dem_staged[slot] = dem_in ? 1 : 0;
    sm.use_stage = fit ? 1 : 0;
    uint32_t bytes = dem_in ? DEM_W * DEM_W * 16 : 0;
    if (fit) bytes += (uint32_t)o4 * 4u * (outs ? 4u : 3u) + (uint32_t)o8 * 8u * 2u;
    tma::fence_proxy_async();  // the CTA's earlier ordinary reads of these bytes come first
    tma::mbar_arrive_expect_tx(&sm.bar, bytes);
    if (dem_in)
        for (int r = 0; r < DEM_W; ++r)
            tma::bulk_g2s(&sm.dem2[slot][r * DEM_W], sh.dem + (int64_t)(ti * TILE + r) * sh.Ny + tj * TILE, DEM_W * 16, &sm.bar);
    if (!fit) return;
    int q4 = 0, q8 = 0;
#pragma unroll
    for (int d = 0; d < 9; ++d) {
        if (n4[d]) {
            tma::bulk_g2s(sm.ts.cell + q4, B.cell + a4[d], n4[d] * 4, &sm.bar);
            tma::bulk_g2s(sm.ts.h + q4, B.h + a4[d], n4[d] * 4, &sm.bar);
            tma::bulk_g2s(sm.ts.m + q4, B.m + a4[d], n4[d] * 4, &sm.bar);
            if (outs) tma::bulk_g2s(sm.ts.vz + q4, B.vz + a4[d], n4[d] * 4, &sm.bar);
            tma::bulk_g2s(sm.ts.f + q8, B.f + a8[d], n8[d] * 8, &sm.bar);
            tma::bulk_g2s(sm.ts.v + q8, B.v + a8[d], n8[d] * 8, &sm.bar);
        }
        q4 += n4[d];
        q8 += n8[d];
    }
}

// P2G quantities of a staged particle (as load_pq)
__device__ __forceinline__ PQ staged_pq(float4 a, float2 v, float vz, int li, int lj, const float4* dem, float g, float hod) {
    PQ p;
    const float4 dm = dem[(li + (a.x >= 1.f ? 1 : 0)) * (TILE + 1) + (lj + (a.y >= 1.f ? 1 : 0))];
    const float K = a.z * g * dm.z * dm.z;
    p.fx = a.x;
    p.fy = a.y;
    p.m = a.z;
    p.mvx = a.z * v.x;
    p.mvy = a.z * v.y;
    p.mh = a.z * a.w;
    p.mvz = a.z * vz;
    p.Kgx = K * dm.x;
    p.Kgy = K * dm.y;
    p.Khh = K * a.w * hod;
    p.li = li;
    p.lj = lj;
    return p;
}

// Sums of one particle over the 3 nodes of stencil rows A0 .. A0+NA-1 of its
// cell (src/simulation.cpp:758-795); OUTS adds m vz. Every operation is
// rounded as written (explicit multiply-adds), so both variants of the cell
// P2G, and any later change of the code around them, sum the same bits.
template <bool OUTS, int A0, int NA>
__device__ __forceinline__ void add_particle_rows(float (&acc)[NA][NQ][3], const PQ& p) {
    float wx[3], wy[3], dwx[3], dwy[3];
    bspline3(p.fx, wx, dwx);
    bspline3(p.fy, wy, dwy);
#pragma unroll
    for (int a = 0; a < NA; ++a) {
        const int A = A0 + a;
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const float wgt = __fmul_rn(wx[A], wy[b]);
            if (wgt > 3e-3f) {  // the reference's weight cut-off (src/simulation.cpp:780)
                acc[a][0][b] = __fmaf_rn(p.m, wgt, acc[a][0][b]);
                acc[a][1][b] = __fmaf_rn(p.mvx, wgt, acc[a][1][b]);
                acc[a][2][b] = __fmaf_rn(p.mvy, wgt, acc[a][2][b]);
                acc[a][3][b] = __fmaf_rn(p.mh, wgt, acc[a][3][b]);
                acc[a][4][b] = __fadd_rn(acc[a][4][b], __fmaf_rn(p.Khh, __fmul_rn(dwx[A], wy[b]), -__fmul_rn(p.Kgx, wgt)));
                acc[a][5][b] = __fadd_rn(acc[a][5][b], __fmaf_rn(p.Khh, __fmul_rn(dwy[b], wx[A]), -__fmul_rn(p.Kgy, wgt)));
                if (OUTS) acc[a][6][b] = __fmaf_rn(p.mvz, wgt, acc[a][6][b]);
            }
        }
    }
}

// Rows A0 .. A0+NA-1 of one cell's particles, summed in sorted order: staged
// in shared memory, or (tiles over P2C_CAP candidates) read through the
// sorted index list in global memory.
template <bool OUTS, int A0, int NA>
__device__ __forceinline__ void cell_row_sums(float (&acc)[NA][NQ][3], bool staged, const P2CSmem& sm, const float4* dem,
                                              const int32_t* order, int c0, int nn, const PBuf& B, int li, int lj, float g,
                                              float hod) {
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int q = 0; q < NQ; ++q)
#pragma unroll
            for (int b = 0; b < 3; ++b) acc[a][q][b] = 0.f;
    if (staged) {
        for (int r = c0; r < c0 + nn; ++r) {
            const int k = sm.idx[r];
            add_particle_rows<OUTS, A0, NA>(acc, staged_pq(sm.st.sa[k], sm.st.sv[k], sm.st.svz[k], li, lj, dem, g, hod));
        }
        return;
    }
    int nsrc = nn > 0 ? order[c0] : 0;
    for (int r = 0; r < nn; ++r) {
        const int src = nsrc;
        if (r + 1 < nn) nsrc = order[c0 + r + 1];
        add_particle_rows<OUTS, A0, NA>(acc, load_pq(B, src, li, lj, dem, g, hod, OUTS));
    }
}

// Stencil rows A0 .. A0+NA-1 of every cell into the node sums: in round
// (A, b) each node receives the row sum of exactly one cell, so the rounds
// need no atomics and every node adds its <= 9 cells in (a, b) order.
template <bool OUTS, int A0, int NA>
__device__ __forceinline__ void p2c_rowset(P2CSmem& sm, bool staged, const float4* dem, const int32_t* order, int c0,
                                           int nn, const PBuf& B, int li, int lj, float g, float hod) {
    float acc[NA][NQ][3];
    cell_row_sums<OUTS, A0, NA>(acc, staged, sm, dem, order, c0, nn, B, li, lj, g, hod);
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            __syncthreads();
            const int nd = (li + A0 + a) * TN + (lj + b);
#pragma unroll
            for (int q = 0; q < (OUTS ? NQ : NQ - 1); ++q) sm.nsum[q * TN * TN + nd] += acc[a][q][b];
        }
}

// Rows per pass over a cell's particles: each pass evaluates the particles'
// weights and quantities once; more rows per pass cost accumulator registers.
#ifndef SLAB_P2C_ROWS
#define SLAB_P2C_ROWS 2
#endif
template <bool OUTS>
__device__ __forceinline__ void p2c_rows(P2CSmem& sm, bool staged, const float4* dem, const int32_t* order, int c0, int nn,
                                         const PBuf& B, int li, int lj, float g, float hod) {
    if constexpr (SLAB_P2C_ROWS == 3) {
        p2c_rowset<OUTS, 0, 3>(sm, staged, dem, order, c0, nn, B, li, lj, g, hod);
    } else if constexpr (SLAB_P2C_ROWS == 2) {
        p2c_rowset<OUTS, 0, 2>(sm, staged, dem, order, c0, nn, B, li, lj, g, hod);
        p2c_rowset<OUTS, 2, 1>(sm, staged, dem, order, c0, nn, B, li, lj, g, hod);
    } else {
        p2c_rowset<OUTS, 0, 1>(sm, staged, dem, order, c0, nn, B, li, lj, g, hod);
        p2c_rowset<OUTS, 1, 1>(sm, staged, dem, order, c0, nn, B, li, lj, g, hod);
        p2c_rowset<OUTS, 2, 1>(sm, staged, dem, order, c0, nn, B, li, lj, g, hod);
    }
}

// K2: P2G of one tile (src/simulation.cpp:726-798) as a segmented reduction
// over cell-sorted particles, with no atomics on floats. The tile's
// descriptor comes from k_prep; then
//  1. the tile's candidates and terrain window come into shared memory as
//     per-thread asynchronous copies, all requested in one round (a tile
//     with more than P2C_CAP candidates reads only their cells, chunk by
//     chunk); then each warp walks a contiguous block of the candidates and
//     counts particles per cell (lanes of one cell are grouped by
//     __match_any_sync);
//  2. thread = cell: per-warp write cursors and the cell's range (a scan);
//  3. the warps walk their blocks again and give each particle its place --
//     a stable counting sort by cell -- as an index in shared memory (large
//     tiles: an index into the tile's segment of the next particle buffer,
//     unused until G2P);
//  4. thread = cell: FP32 sums of the cell's particles, in sorted order, for
//     the 3 nodes of one stencil row at a time (21 accumulators, so 12 tiles
//     fit on an SM), each row added into shared node sums in three rounds:
//     every node adds its <= 9 cells in (a, b) order;
//  5. the node sums are the tile's partial window.
// The candidates of a tile come in an order fixed by the previous step's G2P
// (ordered placement), so every sum has a fixed order: results are bitwise
// reproducible and the same alone or inside a batch. A tile costs one round
// of global loads (its descriptor is read while the tile before it runs);
// each CTA takes a contiguous run of work items.
// With TMA = true the loads of a tile leave its critical path: while tile n
// is summed (phases 2-5), thread 0 has the TMA engine copy tile n+1's
// candidate ranges and terrain window into shared memory (p2c_issue_stage),
// and the descriptor after that is read into registers. Tiles whose
// candidates do not fit the stage load them as before.

// the CTA's scenario values for a run of its tiles (thread 0)
template <typename Sm> __device__ __forceinline__ void p2c_load_scenario(Sm& sm, const Shared& sh, int sid) {
    const Scn& S = sh.scn[sid];
    const SCnt* n = S.cnt;
    const int cur = n->seq & 1;
    sm.B = S.buf[cur];
    sm.nxt_cell = S.buf[cur ^ 1].cell;
    sm.ctl = S.ctl;
    sm.g = S.g;
    sm.hod = 0.5f * S.ood;
    sm.outs = n->outs != 0;
    sm.csid = sid;
}

// thread 0: the copies of the tile in sm.dnext, from its scenario's buffer
__device__ __forceinline__ void p2c_issue_next(P2CSmemTma& sm, const Shared& sh, int slot) {
    const TileDesc& D = sm.dnext;
    if (D.sid == sm.csid) {
        p2c_issue_stage(sm, D, sm.B, sm.outs != 0, sh, slot);
    } else {
        const Scn& S = sh.scn[D.sid];
        const SCnt* n = S.cnt;
        p2c_issue_stage(sm, D, S.buf[n->seq & 1], n->outs != 0, sh, slot);
    }
}

// candidate k of tile D: its range and its position in that range
__device__ __forceinline__ int cand_range(int k, const TileDesc& D, int& off) {
    int d = 0;
    while (d < 8 && D.rpref[d + 1] <= k) ++d;
    off = k - D.rpref[d];
    return d;
}

constexpr int P2C_TMA_MIN_BLOCKS = NCELL == 64 ? 6 : 2;  // the stage doubles the shared memory of a CTA

// 8x8 tiles: a staged candidate's entry in sm.lc packs its local cell (6
// bits) and its rank among the same cell's candidates in its warp's block
// (the rest, up to 511 > P2C_CAP / 2), so the placement needs no warp votes.
constexpr bool P2C_PACKED = NCELL == 64;

// Count one chunk of a warp's candidates per cell: lanes of one cell are
// grouped by __match_any_sync, the group's first lane adds the group to the
// (warp, cell) count; returns each lane's rank among its cell's candidates
// so far in this warp (lc < 0: not in the tile, rank 0).
__device__ __forceinline__ int p2c_count(int (&wcur)[P2C_WARPS][NCELL], int warp, int lane, int lc) {
    const unsigned vm = __ballot_sync(0xffffffffu, lc >= 0);
    int rank = 0;
    if (lc >= 0) {
        const unsigned peers = __match_any_sync(vm, lc);
        const int leader = __ffs(peers) - 1;
        int base = 0;
        if (lane == leader) {
            base = wcur[warp][lc];
            wcur[warp][lc] = base + __popc(peers);
        }
        rank = __shfl_sync(peers, base, leader) + __popc(peers & ((1u << lane) - 1u));
    }
    __syncwarp();
    return rank;
}
// one candidate of phase 1: its range, cell and the quantities to stage
struct P2CCand {
    int d;
    int32_t cell;
    float2 f, v;
    float m, h, vz;
    bool valid;
};

template <bool TMA>
__device__ __forceinline__ void p2g_cell_body(const Shared& sh, int cls, unsigned char* smem_raw, const CUtensorMap* dem_map) {
    using Sm = typename std::conditional<TMA, P2CSmemTma, P2CSmem>::type;
    Sm& sm = *reinterpret_cast<Sm*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const int li = tid / TILE, lj = tid % TILE;
    int i0, i1;
    work_range(p2g_count(sh, cls), i0, i1);
    // the first descriptor now; each later one is read while the tile before it runs
    int w_cur = i0 < i1 ? p2g_item(sh, cls, i0) : 0;
    int w_nxt = i0 + 1 < i1 ? p2g_item(sh, cls, i0 + 1) : 0;
    if (i0 < i1) load_desc(sh.desc + w_cur, &sm.d);
    if (tid == 0) {
        sm.csid = -1;
        if constexpr (TMA) {
            tma::mbar_init(&sm.bar, 1);
        } else {
            tma::mbar_init(&sm.dem_bar, 1);
        }
        tma::fence_mbar_init();
    }
    __syncthreads();
    uint32_t dem_phase = 0;  // parity of the terrain window's next completion
    if constexpr (TMA) {
        if (tid == 0 && i0 < i1) {  // the first tile's copies
            p2c_load_scenario(sm, sh, sm.d.sid);
            sm.dnext = sm.d;
            p2c_issue_next(sm, sh, 0);
        }
    }
    SLAB_PHASE_BEGIN;
    for (int i = i0, n = 0; i < i1; ++i, ++n) {
        const int w = w_cur;
        for (int k = tid; k < P2C_WARPS * NCELL; k += P2C_THREADS) (&sm.wcur[0][0])[k] = 0;
        for (int k = tid; k < NQ * TN * TN; k += P2C_THREADS) sm.nsum[k] = 0.f;
        __syncthreads();
        SLAB_PHASE_MARK(0);
        // the next tile's descriptor (one word per thread) and the item after it
        int dn = 0, w_nn = 0;
        if (i + 1 < i1 && tid < DESC_WORDS) dn = reinterpret_cast<const int*>(sh.desc + w_nxt)[tid];
        if (i + 2 < i1) w_nn = p2g_item(sh, cls, i + 2);
        if (sm.d.sid != sm.csid) {  // uniform: a new scenario in this CTA's run
            __syncthreads();
            if (tid == 0) p2c_load_scenario(sm, sh, sm.d.sid);
            __syncthreads();
        }
        const int t = sm.d.t;
        const int ti = t / sh.TY, tj = t % sh.TY;
        const bool outs = sm.outs != 0;
        Ctl* const ctl = sm.ctl;
        float4* dem;
        bool from_stage = false;
        if constexpr (TMA) {
            const int slot = n & 1;
            dem = sm.dem2[slot];
            if (!tma::mbar_wait(&sm.bar, (uint32_t)(n & 1))) atomicOr(&ctl->err, ERR_TIMEOUT);  // this tile's copies
            from_stage = sm.use_stage != 0;
            if (!sm.dem_staged[slot])
                for (int k = tid; k < DEM_W * DEM_W; k += P2C_THREADS) {
                    const int i = ti * TILE + k / DEM_W, j = tj * TILE + k % DEM_W;
                    dem[k] = (i < sh.Nx && j < sh.Ny) ? sh.dem[(int64_t)i * sh.Ny + j] : make_float4(0.f, 0.f, 1.f, 0.f);
                }
        } else {
            // the terrain window: one 2-D tensor copy (TMA) of its 9 x 9 nodes,
            // issued by one thread, completed before phase 4. The map sees the
            // terrain as [Nx][4 Ny] floats, so x = 4 tj TILE (a multiple of 16
            // bytes). Nodes past the terrain's far edges read as zero; no valid
            // particle uses them (its stencil lies inside the terrain).
            dem = sm.dem;
            if (tid == 0) {
                tma::fence_proxy_async();  // the previous tile's reads of the window come first
                tma::mbar_arrive_expect_tx(&sm.dem_bar, DEM_W * DEM_W * 16);
                tma::tensor_g2s_2d(dem, dem_map, 4 * tj * TILE, ti * TILE, &sm.dem_bar);
            }
        }
        const int ncand = sm.d.rpref[9];
        const int total = sm.d.total;
        const bool staged = ncand <= P2C_CAP;
        const PBuf B = sm.B;
        const int per = (ncand + P2C_WARPS - 1) / P2C_WARPS;
        const int k_lo = min(warp * per, ncand), k_hi = min(k_lo + per, ncand);
        // 1. load (stage) and count per (warp, cell). A warp requests its next
        // chunk of 32 candidates before it stages the current one, so the
        // chunks' load rounds overlap.
        auto load_cand = [&](int k, P2CCand& c) {
            c.valid = k < k_hi;
            c.d = 0;
            c.cell = 0;
            c.f = c.v = make_float2(0.f, 0.f);
            c.m = c.h = c.vz = 0.f;
            if (!c.valid) return;
            if (TMA && from_stage) {  // from the bulk-copied stage
                int off;
                c.d = cand_range(k, sm.d, off);
                if constexpr (TMA) {
                    const int s4 = sm.lead4[c.d] + off, s8 = sm.lead8[c.d] + off;
                    c.cell = sm.ts.cell[s4];
                    c.f = sm.ts.f[s8];
                    c.v = sm.ts.v[s8];
                    c.m = sm.ts.m[s4];
                    c.h = sm.ts.h[s4];
                    if (outs) c.vz = sm.ts.vz[s4];
                }
            } else {
                const int src = cand_to_index(k, sm.d, c.d);
                c.cell = B.cell[src];
                if (staged) {  // issued together with the cell load
                    c.f = B.f[src];
                    c.v = B.v[src];
                    c.m = B.m[src];
                    c.h = B.h[src];
                    if (outs) c.vz = B.vz[src];
                }
            }
        };
        if (!TMA && staged) {
            // every thread requests its share of the tile's candidates (and the
            // terrain window above) as asynchronous copies into the stage: the
            // whole gather is one load round, with no register held per value
            int d = 0;  // range of candidate k: k only grows, so d is carried (rpref[9] = ncand > k bounds it by 8)
            for (int k = tid; k < ncand; k += P2C_THREADS) {
                while (sm.d.rpref[d + 1] <= k) ++d;
                const int src = sm.d.rstart[d] + (k - sm.d.rpref[d]);
                cpa::copy4(&sm.ccell[k], B.cell + src);
                cpa::copy8(&sm.st.sa[k], B.f + src);  // f.x, f.y
                cpa::copy4(&sm.st.sa[k].z, B.m + src);
                cpa::copy4(&sm.st.sa[k].w, B.h + src);
                cpa::copy8(&sm.st.sv[k], B.v + src);
                if (outs) cpa::copy4(&sm.st.svz[k], B.vz + src);
            }
            cpa::wait_all();
            __syncthreads();
            // count per (warp, cell) over the warp's block, as below
            for (int k0 = k_lo; k0 < k_hi; k0 += 32) {
                const int k = k0 + lane;
                int lc = -1;
                if (k < k_hi) {
                    const int32_t cell = sm.ccell[k];
                    const int ci = cell_i(cell) - ti * TILE, cj = cell_j(cell) - tj * TILE;
                    if ((unsigned)ci < TILE && (unsigned)cj < TILE) {
                        lc = ci * TILE + cj;
                    } else {
                        int off;
                        if (cand_range(k, sm.d, off) == 4) atomicOr(&ctl->err, ERR_MOVE);  // a stayer outside its tile
                    }
                }
                const int rank = p2c_count(sm.wcur, warp, lane, lc);
                if (k < k_hi) sm.lc[k] = (int16_t)(lc < 0 ? -1 : (P2C_PACKED ? (rank << 6) | lc : lc));
            }
        } else {
            P2CCand nx;
            load_cand(k_lo + lane, nx);
            for (int k0 = k_lo; k0 < k_hi; k0 += 32) {
                const int k = k0 + lane;
                const P2CCand q = nx;
                if (k0 + 32 < k_hi) load_cand(k0 + 32 + lane, nx);
                int lc = -1;
                if (q.valid) {
                    const int ci = cell_i(q.cell) - ti * TILE, cj = cell_j(q.cell) - tj * TILE;
                    if ((unsigned)ci < TILE && (unsigned)cj < TILE) lc = ci * TILE + cj;
                    else if (q.d == 4) atomicOr(&ctl->err, ERR_MOVE);  // a stayer outside its tile
                    if (staged && lc >= 0) {
                        sm.st.sa[k] = make_float4(q.f.x, q.f.y, q.m, q.h);
                        sm.st.sv[k] = q.v;
                        sm.st.svz[k] = q.vz;
                    }
                }
                const int rank = p2c_count(sm.wcur, warp, lane, lc);
                if (staged && q.valid) sm.lc[k] = (int16_t)(lc < 0 ? -1 : (P2C_PACKED ? (rank << 6) | lc : lc));
            }
        }
        if constexpr (TMA) {
            if (tid < DESC_WORDS) reinterpret_cast<int*>(&sm.dnext)[tid] = dn;
        } else {
            // every thread waits for the terrain window's tensor copy
            if (!tma::mbar_wait(&sm.dem_bar, dem_phase)) atomicOr(&ctl->err, ERR_TIMEOUT);
            dem_phase ^= 1u;
        }
        __syncthreads();
        if constexpr (TMA) {
            // the stage is free: the next tile's copies run beside phases 2-5 of this one
            if (tid == 0 && i + 1 < i1) p2c_issue_next(sm, sh, (n + 1) & 1);
        }
        SLAB_PHASE_MARK(1);
        // 2. cursors: cell-major, warp-minor
        int n_c = 0;
#pragma unroll
        for (int q = 0; q < P2C_WARPS; ++q) {
            const int x = sm.wcur[q][tid];
            sm.wcur[q][tid] = n_c;
            n_c += x;
        }
        const int c0 = block_exclusive_scan(n_c, sm.s_warp);
        if (tid == P2C_THREADS - 1 && c0 + n_c != total) atomicOr(&ctl->err, ERR_CAPACITY);
#pragma unroll
        for (int q = 0; q < P2C_WARPS; ++q) sm.wcur[q][tid] += c0;
        __syncthreads();
        SLAB_PHASE_MARK(2);
        // 3. stable placement by cell: (warp, cell) cursor + rank
        int32_t* order = sm.nxt_cell + sm.d.nxt_off;
        if (P2C_PACKED && staged) {
            for (int k = k_lo + lane; k < k_hi; k += 32) {
                const int e = sm.lc[k];
                if (e >= 0) {
                    const int pos = sm.wcur[warp][e & 63] + (e >> 6);
                    if (pos >= total) atomicOr(&ctl->err, ERR_CAPACITY);
                    else sm.idx[pos] = (int16_t)k;
                }
            }
        } else
        for (int k0 = k_lo; k0 < k_hi; k0 += 32) {
            const int k = k0 + lane;
            int lc = -1, src = 0;
            if (k < k_hi) {
                if (staged) {
                    lc = sm.lc[k];
                } else {
                    int d;
                    src = cand_to_index(k, sm.d, d);
                    const int32_t cell = B.cell[src];
                    const int ci = cell_i(cell) - ti * TILE, cj = cell_j(cell) - tj * TILE;
                    if ((unsigned)ci < TILE && (unsigned)cj < TILE) lc = ci * TILE + cj;
                }
            }
            const unsigned vm = __ballot_sync(0xffffffffu, lc >= 0);
            unsigned peers = 0;
            if (lc >= 0) {
                peers = __match_any_sync(vm, lc);
                const int pos = sm.wcur[warp][lc] + __popc(peers & lt);
                if (pos >= total) atomicOr(&ctl->err, ERR_CAPACITY);
                else if (staged) sm.idx[pos] = (int16_t)k;
                else order[pos] = src;
            }
            __syncwarp();
            if (lc >= 0 && (peers & lt) == 0) sm.wcur[warp][lc] += __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        SLAB_PHASE_MARK(3);
        // 4. per-cell row sums into the node sums
        {
            const int nn = max(0, min(n_c, total - c0));
            const float g = sm.g, hod = sm.hod;
            if (outs) p2c_rows<true>(sm, staged, dem, order, c0, nn, B, li, lj, g, hod);
            else p2c_rows<false>(sm, staged, dem, order, c0, nn, B, li, lj, g, hod);
        }
        __syncthreads();
        SLAB_PHASE_MARK(4);
        // 5. the tile's partial window
        float* P = sh.part + (size_t)w * PART_STRIDE;
        for (int k = tid; k < PART_STRIDE; k += P2C_THREADS) P[k] = sm.nsum[k];
        __syncthreads();
        if (i + 1 < i1 && tid < DESC_WORDS) reinterpret_cast<int*>(&sm.d)[tid] = dn;
        w_cur = w_nxt;
        w_nxt = w_nn;
        SLAB_PHASE_MARK(5);
        SLAB_PHASE_TILE();
    }
    SLAB_PHASE_MARK(6);
    __syncthreads();
    if (tid == 0) {  // every copy was waited for; the memory may serve another purpose next
        if constexpr (TMA) tma::mbar_inval(&sm.bar);
        else tma::mbar_inval(&sm.dem_bar);
    }
}

template <bool TMA>
__global__ void __launch_bounds__(P2C_THREADS, TMA ? P2C_TMA_MIN_BLOCKS : P2C_MIN_BLOCKS)
    k_p2g_cell(Shared sh, int cls, const __grid_constant__ CUtensorMap dem_map) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    p2g_cell_body<TMA>(sh, cls, smem_raw, &dem_map);
}

// ----------------------------------------------------- P2G of sparse tiles

// K2 for tiles with at most split_min particles (src/simulation.cpp:726-798).
// Such a tile's time is load latency, not arithmetic, so the kernel:
//  - keeps the scenario's buffer pointers across consecutive tiles of one
//    scenario, and requests the next tile's descriptor while this one runs;
//  - requests the terrain window and the first candidate of every thread in
//    one round;
//  - pass A: per particle quantities into shared memory, cell counts and the
//    per-quantity bounds of one contribution (as k_p2g);
//  - pass B: one (particle, stencil row) item per thread, three nodes each,
//    added as the hi/lo 32-bit fixed-point pairs of k_p2g<ACC_HILO> with
//    native shared-memory integer atomics. The integer sums are exact, so
//    the result does not depend on arrival order.
constexpr int P2S_THREADS = NCELL;
constexpr int P2S_MIN_BLOCKS = NCELL == 64 ? 16 : 4;
constexpr int P2S_CAP = NCELL;  // particles of a sparse tile (split_min is capped to it)
constexpr int P2S_DEMW = (TILE + 1) * (TILE + 1);
constexpr int P2S_DEM_PER = (P2S_DEMW + P2S_THREADS - 1) / P2S_THREADS;
static_assert(DESC_WORDS <= P2S_THREADS, "one descriptor word per thread");

struct P2SSmem {
    int hi[NQ * TN * TN];  // fixed-point sums of the (TILE+2)^2 window, [q][node]: rounded part
    int lo[NQ * TN * TN];  //                                                      2^-20 finer rest
    float4 dem[P2S_DEMW];
    PQ pq[P2S_CAP];
    int ccnt[NCELL];
    unsigned bmax[NQ];
    int mcc, nv;
    float scale[NQ], iscale[NQ];
    TileDesc d;
};

__device__ __forceinline__ PQ make_pq(float2 f, float2 v, float m, float h, float vz, int li, int lj, const float4* dem, float g, float hod) {
    PQ p;
    const float4 dm = dem[(li + (f.x >= 1.f ? 1 : 0)) * (TILE + 1) + (lj + (f.y >= 1.f ? 1 : 0))];
    const float K = m * g * dm.z * dm.z;
    p.fx = f.x;
    p.fy = f.y;
    p.m = m;
    p.mvx = m * v.x;
    p.mvy = m * v.y;
    p.mh = m * h;
    p.mvz = m * vz;
    p.Kgx = K * dm.x;
    p.Kgy = K * dm.y;
    p.Khh = K * h * hod;
    p.li = li;
    p.lj = lj;
    return p;
}

__device__ __forceinline__ void p2g_sparse_body(const Shared& sh, int cls, unsigned char* smem_raw) {
    P2SSmem& sm = *reinterpret_cast<P2SSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31;
    int i0, i1;
    work_range(p2g_count(sh, cls), i0, i1);
    int w_cur = i0 < i1 ? p2g_item(sh, cls, i0) : 0;
    int w_nxt = i0 + 1 < i1 ? p2g_item(sh, cls, i0 + 1) : 0;
    if (i0 < i1) load_desc(sh.desc + w_cur, &sm.d);
    int csid = -1;
    PBuf B{};
    Ctl* ctl = nullptr;
    bool outs = false;
    float g = 0.f, hod = 0.f;
    for (int i = i0; i < i1; ++i) {
        const int w = w_cur;
        for (int k = tid; k < NQ * TN * TN; k += P2S_THREADS) {
            sm.hi[k] = 0;
            sm.lo[k] = 0;
        }
        for (int k = tid; k < NCELL; k += P2S_THREADS) sm.ccnt[k] = 0;
        if (tid < NQ) sm.bmax[tid] = 0u;
        if (tid == 0) {
            sm.mcc = 0;
            sm.nv = 0;
        }
        __syncthreads();
        // the next tile's descriptor and the item after it, stored at the end
        int dn = 0, w_nn = 0;
        if (i + 1 < i1 && tid < DESC_WORDS) dn = reinterpret_cast<const int*>(sh.desc + w_nxt)[tid];
        if (i + 2 < i1) w_nn = p2g_item(sh, cls, i + 2);
        if (sm.d.sid != csid) {  // uniform: a new scenario in this CTA's run
            csid = sm.d.sid;
            const Scn& S = sh.scn[csid];
            const SCnt* n = S.cnt;
            B = S.buf[n->seq & 1];
            outs = n->outs != 0;
            g = S.g;
            hod = 0.5f * S.ood;
            ctl = S.ctl;
        }
        const int t = sm.d.t;
        const int ti = t / sh.TY, tj = t % sh.TY;
        const int ncand = sm.d.rpref[9];
        // one round: the terrain window and each thread's first candidate
        float4 dmr[P2S_DEM_PER];
#pragma unroll
        for (int r = 0; r < P2S_DEM_PER; ++r) {
            const int k = tid + r * P2S_THREADS;
            const int ii = ti * TILE + k / (TILE + 1), jj = tj * TILE + k % (TILE + 1);
            dmr[r] = (k < P2S_DEMW && ii < sh.Nx && jj < sh.Ny) ? sh.dem[(int64_t)ii * sh.Ny + jj] : make_float4(0.f, 0.f, 1.f, 0.f);
        }
        int d0 = 0;
        int32_t cell0 = 0;
        float2 f0 = make_float2(0.f, 0.f), v0 = make_float2(0.f, 0.f);
        float m0 = 0.f, h0 = 0.f, vz0 = 0.f;
        if (tid < ncand) {
            const int src = cand_to_index(tid, sm.d, d0);
            cell0 = B.cell[src];
            f0 = B.f[src];
            v0 = B.v[src];
            m0 = B.m[src];
            h0 = B.h[src];
            if (outs) vz0 = B.vz[src];
        }
#pragma unroll
        for (int r = 0; r < P2S_DEM_PER; ++r) {
            const int k = tid + r * P2S_THREADS;
            if (k < P2S_DEMW) sm.dem[k] = dmr[r];
        }
        __syncthreads();
        // pass A: particle quantities, cell counts, bounds
        float bm = 0.f, bvx = 0.f, bvy = 0.f, bh = 0.f, bvz = 0.f, bF = 0.f;
        for (int k = tid; k < ncand; k += P2S_THREADS) {
            int d = d0;
            int32_t cell = cell0;
            float2 f = f0, v = v0;
            float m = m0, h = h0, vz = vz0;
            if (k != tid) {
                const int src = cand_to_index(k, sm.d, d);
                cell = B.cell[src];
                f = B.f[src];
                v = B.v[src];
                m = B.m[src];
                h = B.h[src];
                vz = outs ? B.vz[src] : 0.f;
            }
            const int li = cell_i(cell) - ti * TILE, lj = cell_j(cell) - tj * TILE;
            if ((unsigned)li >= TILE || (unsigned)lj >= TILE) {
                if (d == 4) atomicOr(&ctl->err, ERR_MOVE);  // a stayer outside its tile
                continue;
            }
            const PQ p = make_pq(f, v, m, h, vz, li, lj, sm.dem, g, hod);
            const int slot = atomicAdd(&sm.nv, 1);
            if (slot < P2S_CAP) sm.pq[slot] = p;
            else atomicOr(&ctl->err, ERR_CAPACITY);
            const int c = atomicAdd(&sm.ccnt[li * TILE + lj], 1) + 1;
            atomicMax(&sm.mcc, c);
            bm = fmaxf(bm, p.m);
            bvx = fmaxf(bvx, fabsf(p.mvx));
            bvy = fmaxf(bvy, fabsf(p.mvy));
            bh = fmaxf(bh, p.mh);
            bvz = fmaxf(bvz, fabsf(p.mvz));
            bF = fmaxf(bF, p.Khh + fmaxf(fabsf(p.Kgx), fabsf(p.Kgy)));
        }
        bm = warp_max(bm);
        bvx = warp_max(bvx);
        bvy = warp_max(bvy);
        bh = warp_max(bh);
        bvz = warp_max(bvz);
        bF = warp_max(bF);
        if (lane == 0) {
            atomicMax(&sm.bmax[0], __float_as_uint(bm));
            atomicMax(&sm.bmax[1], __float_as_uint(bvx));
            atomicMax(&sm.bmax[2], __float_as_uint(bvy));
            atomicMax(&sm.bmax[3], __float_as_uint(bh));
            atomicMax(&sm.bmax[4], __float_as_uint(bF));
            atomicMax(&sm.bmax[5], __float_as_uint(bF));
            atomicMax(&sm.bmax[6], __float_as_uint(bvz));
        }
        __syncthreads();
        if (tid < NQ) {
            const float bound = 9.f * (float)sm.mcc * 0.75f * __uint_as_float(sm.bmax[tid]);
            int e = 0;
            if (bound > 0.f) {
                int E;
                frexpf(bound, &E);  // bound < 2^E
                e = min(max(30 - E, -120), 120);
            }
            sm.scale[tid] = ldexpf(1.f, e);
            sm.iscale[tid] = ldexpf(1.f, -e);
        }
        __syncthreads();
        // pass B: (particle, stencil row) items
        const int nv = min(sm.nv, P2S_CAP);
        const int lob = lo_bits_for(9 * sm.mcc);  // lo sums of a node stay below 2^30 (20 bits for <= 64 particles)
        const float lo_mul = ldexpf(1.f, lob);
        const double lo_div = ldexp(1.0, -lob);
        for (int it = tid; it < 3 * nv; it += P2S_THREADS) {
            const int pi = it / 3, a = it - 3 * pi;
            const PQ p = sm.pq[pi];
            float wx[3], wy[3], dwx[3], dwy[3];
            bspline3(p.fx, wx, dwx);
            bspline3(p.fy, wy, dwy);
            const float wxa = a == 0 ? wx[0] : (a == 1 ? wx[1] : wx[2]);
            const float dwxa = a == 0 ? dwx[0] : (a == 1 ? dwx[1] : dwx[2]);
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const float wgt = wxa * wy[b];
                if (wgt > 3e-3f) {  // the reference's weight cut-off (src/simulation.cpp:780)
                    const int nd = (p.li + a) * TN + (p.lj + b);
                    const float cq[NQ] = {p.m * wgt, p.mvx * wgt, p.mvy * wgt, p.mh * wgt, p.Khh * (dwxa * wy[b]) - p.Kgx * wgt,
                                          p.Khh * (dwy[b] * wxa) - p.Kgy * wgt, p.mvz * wgt};
#pragma unroll
                    for (int q = 0; q < NQ; ++q) {
                        if (q == 6 && !outs) continue;
                        const float x = cq[q] * sm.scale[q];
                        const int h_ = __float2int_rn(x);
                        atomicAdd(sm.hi + q * TN * TN + nd, h_);
                        const int l_ = __float2int_rn((x - (float)h_) * lo_mul);
                        if (l_) atomicAdd(sm.lo + q * TN * TN + nd, l_);
                    }
                }
            }
        }
        __syncthreads();
        float* P = sh.part + (size_t)w * PART_STRIDE;
        for (int k = tid; k < PART_STRIDE; k += P2S_THREADS)
            P[k] = (float)(((double)sm.hi[k] + (double)sm.lo[k] * lo_div) * (double)sm.iscale[k / (TN * TN)]);
        __syncthreads();
        if (i + 1 < i1 && tid < DESC_WORDS) reinterpret_cast<int*>(&sm.d)[tid] = dn;
        w_cur = w_nxt;
        w_nxt = w_nn;
    }
}

__global__ void __launch_bounds__(P2S_THREADS, P2S_MIN_BLOCKS) k_p2g_sparse(Shared sh, int cls) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    p2g_sparse_body(sh, cls, smem_raw);
}

// ------------------------------------------------------------ grid update

// Values of one scenario that the grid update reads for every grid tile.
struct GridScn {
    SCnt* n;
    Ctl* c;
    int32_t* act_stamp;
    int32_t* slot_of;
    int32_t* blk_of;
    float dt, g, mu_c, mu_v, xi, mu1, mu2, I0, d, phi;
    int sid, seq, stepid, outs, fric;
};

__device__ __forceinline__ void load_grid_scn(const Shared& sh, int sid, GridScn& z) {
    const Scn& S = sh.scn[sid];
    SCnt* n = S.cnt;
    z.n = n;
    z.c = S.ctl;
    z.act_stamp = S.act_stamp;
    z.slot_of = S.slot_of;
    z.blk_of = S.blk_of;
    z.dt = (float)S.ctl->dt;
    z.g = S.g;
    z.mu_c = S.mu_c;
    z.mu_v = S.mu_v;
    z.xi = S.xi;
    z.mu1 = S.mu1;
    z.mu2 = S.mu2;
    z.I0 = S.I0;
    z.d = S.d;
    z.phi = S.phi;
    z.fric = S.fric;
    z.sid = sid;
    z.seq = n->seq;
    z.stepid = n->stepid;
    z.outs = n->outs;
}

// K3 + K6: computeGridVelocity (src/simulation.cpp:800-875) for the TILE^2
// nodes owned by one grid tile. A node's P2G sum is the partials of the
// tiles whose window covers it, added in a fixed order (own, -x, -y, -xy).
// h_max / v_max2 are updated in the node block; the FP64 grid mass sum is
// the conservation diagnostic.
// Latency: the scenario's values stay in shared memory across a run of its
// grid tiles, and thread 0 reads the grid-tile list two entries ahead.
__device__ __forceinline__ void grid_body(const Shared& sh) {
    __shared__ int s_gt, s_blk;
    __shared__ int s_slot[4];
    __shared__ double s_red[NCELL / 32];
    __shared__ unsigned s_act[NCELL / 32];
    __shared__ GridScn Z;
    const int tid = threadIdx.x;
    const int li = tid / TILE, lj = tid % TILE;
    int w0, w1;
    work_range(min(*sh.gcount, sh.gcap), w0, w1);
    // thread 0: the current and the next entry of the flat grid-tile list
    int2 e_cur = make_int2(-1, 0), e_nxt = make_int2(-1, 0);
    if (tid == 0) {
        Z.sid = -1;
        if (w0 < w1) e_cur = reinterpret_cast<const int2*>(sh.gflat)[w0];
        if (w0 + 1 < w1) e_nxt = reinterpret_cast<const int2*>(sh.gflat)[w0 + 1];
    }
    for (int w = w0; w < w1; ++w) {
        if (tid == 0) {
            if (e_cur.x != Z.sid) load_grid_scn(sh, e_cur.x, Z);  // a new scenario in this CTA's run
            s_gt = e_cur.y;
            e_cur = e_nxt;
            if (w + 2 < w1) e_nxt = reinterpret_cast<const int2*>(sh.gflat)[w + 2];
        }
        __syncthreads();
        Ctl* c = Z.c;
        const int gt = s_gt;
        const int gi = gt / sh.TY, gj = gt % sh.TY;
        if (tid < 4) {
            // contributor k: tile (gi - (k>>1), gj - (k&1)); slot if active this step
            const int ti_ = gi - (tid >> 1), tj_ = gj - (tid & 1);
            int slot = -1;
            if (ti_ >= 0 && tj_ >= 0) {
                const int tt = ti_ * sh.TY + tj_;
                const int st_ = Z.act_stamp[tt], sl = Z.slot_of[tt];  // both loads in flight together
                if (st_ == Z.seq) slot = sl;
            }
            s_slot[tid] = slot;
        } else if (tid == 32) {
            int blk = Z.blk_of[gt];
            if (blk < 0) {
                // a block released by a retired scenario, else a fresh one
                const int f = atomicSub(sh.free_count, 1);
                if (f > 0) {
                    blk = sh.free_blocks[f - 1];
                } else {
                    atomicAdd(sh.free_count, 1);
                    blk = atomicAdd(sh.blk_count, 1);
                }
                if (blk >= sh.blk_cap) {
                    atomicOr(&c->err, ERR_CAPACITY);
                    blk = -1;
                } else {
                    Z.blk_of[gt] = blk;
                    sh.blk_owner[blk] = Z.sid;
                }
            }
            if (blk >= 0) sh.blk_stamp[blk] = Z.stepid;
            s_blk = blk;
        }
        __syncthreads();
        const int blk = s_blk;
        // the block of this grid tile is entry k of contributor k's window (for G2P)
        if (tid < 4 && s_slot[tid] >= 0) sh.desc[s_slot[tid]].blk4[tid] = blk;
        double mloc = 0.0;
        if (blk >= 0) {
            float q[NQ];
#pragma unroll
            for (int k = 0; k < NQ; ++k) q[k] = 0.f;
            auto add = [&](int slot, int a, int b) {
                if (slot < 0) return;
                const float* P = sh.part + (size_t)slot * PART_STRIDE + a * TN + b;
#pragma unroll
                for (int k = 0; k < NQ; ++k) q[k] += P[k * TN * TN];
            };
            const int i = gi * TILE + li, j = gj * TILE + lj;
            const size_t bn = (size_t)blk * NCELL + tid;
            const bool inside = i < sh.Nx && j < sh.Ny;
            // terrain and maxima are requested with the partials (one round of loads)
            const float4 dm = inside ? sh.dem[(int64_t)i * sh.Ny + j] : make_float4(0.f, 0.f, 1.f, 0.f);
            const float hmax0 = sh.hmax[bn], vmax0 = sh.vmax2[bn];
            add(s_slot[0], li, lj);
            if (li < 2) add(s_slot[2], li + TILE, lj);
            if (lj < 2) add(s_slot[1], li, lj + TILE);
            if (li < 2 && lj < 2) add(s_slot[3], li + TILE, lj + TILE);
            float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
            float hn = 0.f, vzn = 0.f;
            const float mi = q[0];
            if (mi > 1e-6f && inside) {
                const float vox = q[1] / mi, voy = q[2] / mi;
                vzn = q[6] / mi;
                hn = q[3] / mi;
                const float dt = Z.dt;
                const float vtx = vox + dt * (q[4] / mi), vty = voy + dt * (q[5] / mi);
                const float vsq = vtx * vtx + vty * vty;
                float nvx = 0.f, nvy = 0.f;
                if (vsq > 1e-16f) {
                    const float ct = dm.z;
                    const float vz = vtx * dm.x + vty * dm.y;
                    const float v3sq = vsq + vz * vz;
                    const float v3 = sqrtf(v3sq);
                    const float g = Z.g;
                    float af;
                    if (Z.fric == SLAB_COULOMB) {
                        af = Z.mu_c * g * ct;
                    } else if (Z.fric == SLAB_VOELLMY) {
                        af = Z.mu_v * g * ct + g * v3sq / (Z.xi * hn * ct);
                    } else {
                        const float I = 5.f * Z.d * v3 / (2.f * hn * ct * ct * sqrtf(g * hn * Z.phi));
                        const float muI = Z.mu1 + (Z.mu2 - Z.mu1) / (1.f + Z.I0 / I);
                        af = muI * g * ct;
                    }
                    const float dv = dt * af;
                    if (dv < v3) {
                        const float fct = 1.f - dv / v3;
                        nvx = vtx * fct;
                        nvy = vty * fct;
                    }
                }
                out = make_float4(nvx, nvy, nvx - vox, nvy - voy);
                sh.hmax[bn] = fmaxf(hmax0, hn);
                sh.vmax2[bn] = fmaxf(vmax0, nvx * nvx + nvy * nvy);
                mloc = (double)mi;
            }
            sh.nv[bn] = out;
            if (Z.outs) {
                sh.oh[bn] = hn;
                sh.om[bn] = inside ? mi : 0.f;
                sh.ovz[bn] = vzn;
                sh.oFx[bn] = inside ? q[4] : 0.f;
                sh.oFy[bn] = inside ? q[5] : 0.f;
            }
        }
        // FP64 grid mass and active-node count of this tile (fixed-order block reduction)
        const unsigned act = __popc(__ballot_sync(0xffffffffu, mloc != 0.0));
        for (int o = 16; o > 0; o >>= 1) mloc += __shfl_xor_sync(0xffffffffu, mloc, o);
        if ((tid & 31) == 0) {
            s_red[tid >> 5] = mloc;
            s_act[tid >> 5] = act;
        }
        __syncthreads();
        if (tid == 0) {
            double sum = 0.0;
            unsigned na = 0;
            for (int k = 0; k < NCELL / 32; ++k) {
                sum += s_red[k];
                na += s_act[k];
            }
            if (sum != 0.0) atomicAdd(&Z.n->grid_mass, sum);
            if (na) atomicAdd(&c->node_steps, (unsigned long long)na);
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(NCELL) k_grid(Shared sh) { grid_body(sh); }

// -------------------------------------------------------------------- G2P

__device__ __forceinline__ int dir_of(int ib, int jb, int ti, int tj) {
    int di = (ib >= 0 ? ib / TILE : -1) - ti, dj = (jb >= 0 ? jb / TILE : -1) - tj;
    if (di < -1 || di > 1 || dj < -1 || dj > 1) return -1;
    return (di + 1) * 3 + (dj + 1);
}

#ifndef SLAB_G2P_MIN_BLOCKS
#define SLAB_G2P_MIN_BLOCKS (NCELL == 64 ? 14 : 3)
#endif
constexpr int G2P_MIN_BLOCKS = SLAB_G2P_MIN_BLOCKS;  // resident G2P CTAs per SM the register budget is cut for

// Values of one scenario that a G2P launch reads for every tile: loaded
// once per run of consecutive tiles of that scenario.
struct G2PScn {
    SCnt* n;
    Ctl* c;
    PBuf B, O;                 // current and next particle buffers
    int32_t* grp_nxt;          // segment records of the next step
    int32_t* act_stamp;
    int32_t* act_list_nxt;
    int32_t* act_count_nxt;
    double dx;
    float dt, dt_ood, ood, fr;
    int sid, seq, act_cap, outs, need_vz;
};

__device__ __forceinline__ void load_g2p_scn(const Shared& sh, int sid, G2PScn& z) {
    const Scn& S = sh.scn[sid];
    SCnt* n = S.cnt;
    Ctl* c = S.ctl;
    const int seq = n->seq, cur = seq & 1, nxt = cur ^ 1;
    z.n = n;
    z.c = c;
    z.B = S.buf[cur];
    z.O = S.buf[nxt];
    z.grp_nxt = S.grp[nxt];
    z.act_stamp = S.act_stamp;
    z.act_list_nxt = S.act_list[nxt];
    z.act_count_nxt = &n->act_count[nxt];
    z.dx = c->dx;
    z.dt = (float)c->dt;
    z.ood = S.ood;
    z.dt_ood = z.dt * S.ood;
    z.fr = S.fr;
    z.sid = sid;
    z.seq = seq;
    z.act_cap = S.act_cap;
    z.outs = n->outs != 0;
    z.need_vz = z.outs || n->vz_next;
}

// puts tile tt on the next step's active list, once
__device__ __forceinline__ void g2p_activate(const G2PScn& z, int tt) {
    if (atomicMax(&z.act_stamp[tt], z.seq + 1) < z.seq + 1) {
        const int kk = atomicAdd(z.act_count_nxt, 1);
        if (kk < z.act_cap) z.act_list_nxt[kk] = tt;
        else atomicOr(&z.c->err, ERR_CAPACITY);
    }
}

#ifndef SLAB_G2P_CAP
#define SLAB_G2P_CAP (NCELL == 64 ? 5 * NCELL : 4 * NCELL)
#endif
constexpr int G2P_CAP = SLAB_G2P_CAP;  // candidates of a tile staged in shared memory (more are loaded chunk by chunk)

// a tile's candidates, by candidate index
struct G2PStage {
    float2 f[G2P_CAP];
    float2 v[G2P_CAP];
    int32_t cell[G2P_CAP];
    float h[G2P_CAP];
    float m[G2P_CAP];
    int32_t id[G2P_CAP];
};

struct G2PSmem {
    G2PStage st;
    float4 nv[TN * TN];
    float4 dem[(TILE + 1) * (TILE + 1)];
    int front, back;
    int wst[2][NCELL / 32], wmv[2][NCELL / 32];  // per-warp stayer / mover counts of a chunk (double buffered)
    int dcnt[9];
    TileDesc d;
    G2PScn z;
    double red[5][NCELL / 32];
};

// one candidate of a tile in G2P: its index, data, and whether it is in the tile
struct G2PCand {
    int src;
    int32_t cell, pid;
    float2 f, v;
    float h, m;
    bool valid;
};

__device__ __forceinline__ G2PCand load_g2p_cand(const TileDesc& D, const PBuf& B, int k, int ncand, int t, int TY) {
    G2PCand q;
    q.valid = k < ncand;
    q.src = 0;
    q.cell = 0;
    q.pid = 0;
    q.f = make_float2(1.f, 1.f);
    q.v = make_float2(0.f, 0.f);
    q.h = q.m = 0.f;
    if (q.valid) {
        int r;
        q.src = cand_to_index(k, D, r);
        q.cell = B.cell[q.src];  // the other loads go out with it; the filter is applied on use
        q.f = B.f[q.src];
        q.v = B.v[q.src];
        q.h = B.h[q.src];
        q.m = B.m[q.src];
        q.pid = B.id[q.src];
        q.valid = tile_of_cell(q.cell, TY) == t;
    }
    return q;
}

// candidate k of the tile from the stage (as load_g2p_cand)
__device__ __forceinline__ G2PCand staged_g2p_cand(const G2PStage& st, int k, int ncand, int t, int TY) {
    G2PCand q;
    q.valid = k < ncand;
    q.src = 0;
    q.cell = 0;
    q.pid = 0;
    q.f = make_float2(1.f, 1.f);
    q.v = make_float2(0.f, 0.f);
    q.h = q.m = 0.f;
    if (q.valid) {
        q.cell = st.cell[k];
        q.f = st.f[k];
        q.v = st.v[k];
        q.h = st.h[k];
        q.m = st.m[k];
        q.pid = st.id[k];
        q.valid = tile_of_cell(q.cell, TY) == t;
    }
    return q;
}

// K4: G2P (src/simulation.cpp:877-940) of one tile: FLIP/PIC blend,
// advection, depth update, and the write of the particle into the tile's
// segment of the next buffer -- stayers from the front, particles that moved
// to a neighbour tile from the back, with per-direction counts. The block
// max of |v|^2 and the particle bounding box feed the next step's dt and
// remesh box (K5). Latency: the scenario's values stay in shared memory
// across a run of its tiles, the next tile's descriptor is requested while
// this one runs, a tile's candidates (up to G2P_CAP), node window and terrain
// come into shared memory by asynchronous copies requested in one round, and
// a tile's neighbour activations (two dependent atomics) are issued while the
// next tile's copies are in flight.
__device__ __forceinline__ void g2p_body(const Shared& sh, const double* __restrict__ z64, G2PSmem& sm) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nwork = sh.work_pref[sh.nscn];
    int w0, w1;
    work_range(nwork, w0, w1);
    if (w0 < w1) load_desc(sh.desc + w0, &sm.d);
    if (tid == 0) sm.z.sid = -1;
    int pend_tt = -1;  // threads 0..8: neighbour tile the previous tile activates
    SLAB_PHASE_BEGIN;
    for (int w = w0; w < w1; ++w) {
        if (tid < 9) sm.dcnt[tid] = 0;
        __syncthreads();
        SLAB_PHASE_MARK(8);
        int dn = 0;
        if (w + 1 < w1 && tid < DESC_WORDS) dn = reinterpret_cast<const int*>(sh.desc + w + 1)[tid];
        if (sm.d.sid != sm.z.sid) {  // uniform: a new scenario in this CTA's run
            if (pend_tt >= 0) g2p_activate(sm.z, pend_tt);
            pend_tt = -1;
            __syncthreads();
            if (tid == 0) load_g2p_scn(sh, sm.d.sid, sm.z);
            __syncthreads();
        }
        const G2PScn& Z = sm.z;
        Ctl* c = Z.c;
        const int t = sm.d.t;
        const int ti = t / sh.TY, tj = t % sh.TY;
        const bool outs = Z.outs != 0;
        const bool need_vz = Z.need_vz != 0;
        const int ncand = sm.d.rpref[9];
        const bool staged = ncand <= G2P_CAP;
        // the tile's candidates (the first chunk's, for a tile over the stage),
        // the node window and the terrain are requested together; the stage
        // and the windows fill by asynchronous copies
        G2PCand pre = {};
        if (staged) {
            const PBuf& B = Z.B;
            for (int k = tid; k < ncand; k += NCELL) {
                int r;
                const int src = cand_to_index(k, sm.d, r);
                cpa::copy8(&sm.st.f[k], B.f + src);
                cpa::copy8(&sm.st.v[k], B.v + src);
                cpa::copy4(&sm.st.cell[k], B.cell + src);
                cpa::copy4(&sm.st.h[k], B.h + src);
                cpa::copy4(&sm.st.m[k], B.m + src);
                cpa::copy4(&sm.st.id[k], B.id + src);
            }
        } else {
            pre = load_g2p_cand(sm.d, Z.B, tid, ncand, t, sh.TY);
        }
        // the node window by per-thread asynchronous copies; a part whose grid tile
        // has no block this step (or past the terrain edge) is zero. (Bulk copies
        // of the blocks' rows, issued by warp 0 on an mbarrier, gave the same
        // bits but made the kernel 6 % slower.)
        for (int k = tid; k < TN * TN; k += NCELL) {
            const int a = k / TN, b = k % TN;
            const int i = ti * TILE + a, j = tj * TILE + b;
            const int blk = (i < sh.Nx && j < sh.Ny) ? sm.d.blk4[(a >= TILE ? 2 : 0) + (b >= TILE ? 1 : 0)] : -1;
            if (blk >= 0) cpa::copy16(&sm.nv[k], &sh.nv[(size_t)blk * NCELL + (a % TILE) * TILE + (b % TILE)]);
            else sm.nv[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        if (need_vz) {
            for (int k = tid; k < (TILE + 1) * (TILE + 1); k += NCELL) {
                const int i = ti * TILE + k / (TILE + 1), j = tj * TILE + k % (TILE + 1);
                if (i < sh.Nx && j < sh.Ny) cpa::copy16(&sm.dem[k], sh.dem + (int64_t)i * sh.Ny + j);
                else sm.dem[k] = make_float4(0.f, 0.f, 1.f, 0.f);
            }
        }
        if (pend_tt >= 0) g2p_activate(Z, pend_tt);  // the previous tile's, while the loads above are in flight
        pend_tt = -1;
        SLAB_PHASE_MARK(9);
        cpa::wait_all();
        __syncthreads();
        SLAB_PHASE_MARK(10);
        const int total = sm.d.total;
        const int base = sm.d.nxt_off;
        const PBuf& B = Z.B;
        const PBuf O = Z.O;
        const float dt = Z.dt;
        const float dt_ood = Z.dt_ood;
        const double dx = Z.dx;
        double mnx = INFINITY, mxx = 0.0, mny = INFINITY, mxy = 0.0, vv = 0.0;
        int front = 0, back = 0;  // stayers / movers placed so far (same in every thread)
        G2PCand nxt = pre;
        for (int k0 = 0; k0 < ncand; k0 += NCELL) {
            // this chunk's candidates, and the next chunk's requested before this one is computed
            G2PCand q;
            if (staged) {
                q = staged_g2p_cand(sm.st, k0 + tid, ncand, t, sh.TY);
            } else {
                q = nxt;
                if (k0 + NCELL < ncand) nxt = load_g2p_cand(sm.d, B, k0 + NCELL + tid, ncand, t, sh.TY);
            }
            const bool valid = q.valid;
            const int32_t cell = q.cell;
            int d = 4, ib = 0, jb = 0;
            float2 fn = make_float2(1.f, 1.f), vn = make_float2(0.f, 0.f);
            float hn = 0.f, m = 0.f, vzp = 0.f;
            double zp = 0.0;
            int32_t pid = 0;
            if (valid) {
                const float2 f = q.f;
                const float2 v = q.v;
                const float h = q.h;
                m = q.m;
                pid = q.pid;
                const int ci = cell_i(cell) - ti * TILE, cj = cell_j(cell) - tj * TILE;
                float wx[3], wy[3], dwx[3], dwy[3];
                bspline3(f.x, wx, dwx);
                bspline3(f.y, wy, dwy);
                float picx = 0.f, picy = 0.f, flx = 0.f, fly = 0.f, div = 0.f;
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int b = 0; b < 3; ++b) {
                        const float wgt = wx[a] * wy[b];
                        const float4 nv = sm.nv[(ci + a) * TN + (cj + b)];
                        picx += nv.x * wgt;
                        picy += nv.y * wgt;
                        flx += nv.z * wgt;
                        fly += nv.w * wgt;
                        div += (dwx[a] * wy[b]) * nv.x + (dwy[b] * wx[a]) * nv.y;
                    }
                div *= Z.ood;
                const float fr = Z.fr;
                vn = make_float2(fr * (v.x + flx) + (1.f - fr) * picx, fr * (v.y + fly) + (1.f - fr) * picy);
                hn = h / (1.f + dt * div);
                if (need_vz) {
                    const float4 dm = sm.dem[(ci + (f.x >= 1.f ? 1 : 0)) * (TILE + 1) + (cj + (f.y >= 1.f ? 1 : 0))];
                    vzp = vn.x * dm.x + vn.y * dm.y;
                }
                if (outs) {
                    const int i0 = cell_i(cell), j0 = cell_j(cell);
#pragma unroll
                    for (int a = 0; a < 3; ++a)
#pragma unroll
                        for (int b = 0; b < 3; ++b) zp += (double)(wx[a] * wy[b]) * z64[(int64_t)(i0 + a) * sh.Ny + (j0 + b)];
                }
                // advection with the PIC velocity and re-anchoring of the offset
                const float ux = f.x + dt_ood * picx, uy = f.y + dt_ood * picy;
                const int ki = (int)floorf(ux - 0.5f), kj = (int)floorf(uy - 0.5f);
                ib = cell_i(cell) + ki;
                jb = cell_j(cell) + kj;
                fn = make_float2(ux - (float)ki, uy - (float)kj);
                d = dir_of(ib, jb, ti, tj);
                if (d < 0) {
                    atomicOr(&c->err, ERR_MOVE);
                    d = 4;
                }
                if (ib < 0 || jb < 0 || ib + 2 > sh.Nx - 1 || jb + 2 > sh.Ny - 1) {
                    atomicOr(&c->err, ERR_DOMAIN);
                    ib = min(max(ib, 0), sh.Nx - 3);
                    jb = min(max(jb, 0), sh.Ny - 3);
                    d = dir_of(ib, jb, ti, tj);
                    if (d < 0) d = 4;
                }
                const double px = ((double)ib + (double)fn.x) * dx, py = ((double)jb + (double)fn.y) * dx;
                mnx = fmin(mnx, px);
                mxx = fmax(mxx, px);
                mny = fmin(mny, py);
                mxy = fmax(mxy, py);
                vv = fmax(vv, (double)(vn.x * vn.x + vn.y * vn.y));
                if (!isfinite(vn.x) || !isfinite(vn.y) || !isfinite(hn) || !isfinite(fn.x) || !isfinite(fn.y))
                    atomicOr(&c->err, ERR_NONFINITE);
            }
            // stayers to the front of the segment, movers to the back, both in
            // candidate order (a block prefix of the warps' counts), so the next
            // step sees the tile's particles in an order fixed by the data
            const bool stay = valid && d == 4, move = valid && d != 4;
            const unsigned ms = __ballot_sync(0xffffffffu, stay), mm = __ballot_sync(0xffffffffu, move);
            const int par = (k0 / NCELL) & 1;
            if (lane == 0) {
                sm.wst[par][warp] = __popc(ms);
                sm.wmv[par][warp] = __popc(mm);
            }
            __syncthreads();
            int bs = front, bm = back;
#pragma unroll
            for (int q = 0; q < NCELL / 32; ++q) {
                const int a = sm.wst[par][q], b = sm.wmv[par][q];
                if (q < warp) {
                    bs += a;
                    bm += b;
                }
                front += a;
                back += b;
            }
            const unsigned lt = (1u << lane) - 1u;
            if (valid) {
                int pos;
                if (stay) {
                    pos = base + bs + __popc(ms & lt);
                } else {
                    pos = base + total - 1 - (bm + __popc(mm & lt));
                    atomicAdd(&sm.dcnt[d], 1);
                }
                O.cell[pos] = pack_cell(ib, jb);
                O.f[pos] = fn;
                O.v[pos] = vn;
                O.h[pos] = hn;
                O.m[pos] = m;
                O.id[pos] = pid;
                if (need_vz) O.vz[pos] = vzp;
                if (outs) O.z[pos] = (float)zp;
            }
        }
        SLAB_PHASE_MARK(11);
        if (tid == 0) {
            sm.front = front;
            sm.back = back;
        }
        __syncthreads();
        if (tid < 9) {
            int32_t* G = Z.grp_nxt + (size_t)t * GRP_STRIDE;
            const int cnt = tid == 4 ? sm.front : sm.dcnt[tid];
            G[3 + tid] = cnt;
            if (tid == 0) {
                G[0] = base;
                G[1] = base + sm.front;
                G[2] = base + sm.front + sm.back;
                G[GRP_STAMP] = Z.seq + 1;
                if (sm.front + sm.back != total) atomicOr(&c->err, ERR_CAPACITY);
            }
            if (cnt) pend_tt = (ti + dir_i(tid)) * sh.TY + (tj + dir_j(tid));
        }
        // per-tile reductions into the scenario's control block
        mnx = warp_min(mnx);
        mxx = warp_max(mxx);
        mny = warp_min(mny);
        mxy = warp_max(mxy);
        vv = warp_max(vv);
        if (lane == 0) {
            sm.red[0][warp] = mnx;
            sm.red[1][warp] = mxx;
            sm.red[2][warp] = mny;
            sm.red[3][warp] = mxy;
            sm.red[4][warp] = vv;
        }
        __syncthreads();
        if (tid == 0 && total > 0) {
            for (int k = 1; k < NCELL / 32; ++k) {
                mnx = fmin(mnx, sm.red[0][k]);
                mxx = fmax(mxx, sm.red[1][k]);
                mny = fmin(mny, sm.red[2][k]);
                mxy = fmax(mxy, sm.red[3][k]);
                vv = fmax(vv, sm.red[4][k]);
            }
            atomicMin(reinterpret_cast<unsigned long long*>(&c->pos_acc[0]), (unsigned long long)__double_as_longlong(mnx));
            atomicMax(reinterpret_cast<unsigned long long*>(&c->pos_acc[1]), (unsigned long long)__double_as_longlong(mxx));
            atomicMin(reinterpret_cast<unsigned long long*>(&c->pos_acc[2]), (unsigned long long)__double_as_longlong(mny));
            atomicMax(reinterpret_cast<unsigned long long*>(&c->pos_acc[3]), (unsigned long long)__double_as_longlong(mxy));
            atomicMax(reinterpret_cast<unsigned long long*>(&c->vmax2_acc), (unsigned long long)__double_as_longlong(vv));
        }
        __syncthreads();
        if (w + 1 < w1 && tid < DESC_WORDS) reinterpret_cast<int*>(&sm.d)[tid] = dn;
        SLAB_PHASE_MARK(12);
        SLAB_PHASE_TILE_G2P();
    }
    if (pend_tt >= 0) g2p_activate(sm.z, pend_tt);  // the last tile's
}

__global__ void __launch_bounds__(NCELL, G2P_MIN_BLOCKS) k_g2p(Shared sh, const double* __restrict__ z64) {
    __shared__ G2PSmem sm;
    g2p_body(sh, z64, sm);
}

// K5: end of the step for every running scenario (the per-step reductions
// of G2P into dt, time and the remesh box), then the next step's dt, stop
// rules and work list. One CTA, after G2P.
__device__ __forceinline__ void end_body(const Shared& sh) {
    for (int s = threadIdx.x; s < sh.nscn; s += blockDim.x) {
        const Scn& S = sh.scn[s];
        Ctl* c = S.ctl;
        if (!c->active) continue;
        SCnt* n = S.cnt;
        if (n->cursor != S.Np) atomicOr(&c->err, ERR_CAPACITY);
        ctl_end(c);
        n->seq += 1;
        n->vz_valid = n->outs;
    }
    __syncthreads();
    begin_scenarios(sh, 0);
}

__global__ void k_end(Shared sh) { end_body(sh); }

// ------------------------------------------------------- persistent steps

// Barrier of the persistent step kernel: one cooperative launch, every CTA
// resident. Thread 0 of each CTA arrives on the counter; the last arrival
// resets it and advances the generation; the others wait for the generation
// to change -- at most `limit` clock cycles, after which the CTA records
// ERR_TIMEOUT in every scenario's control block and leaves the kernel. A CTA
// that left never arrives again, so every later wait of the launch runs out
// too: the launch always ends, and no phase runs on inputs that a phase
// before it did not finish (a phase starts only when every CTA arrived).
// The engine is then dead: its later persistent launches return at once.
struct GridBar {
    unsigned count;
    unsigned gen;
    int dead;  // a wait ran out: this engine's step state is incomplete, later launches do nothing
    int pad_;
};

__device__ __forceinline__ bool grid_sync(const Shared& sh, GridBar* bar, long long limit) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        volatile unsigned* vgen = &bar->gen;
        const unsigned g = *vgen;
        __threadfence();
        if (atomicAdd(&bar->count, 1u) == gridDim.x - 1) {
            *reinterpret_cast<volatile unsigned*>(&bar->count) = 0u;
            __threadfence();
            atomicAdd(&bar->gen, 1u);
        } else {
            const long long t0 = clock64();
            while (*vgen == g) {
                if (clock64() - t0 > limit) {
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
            if (!ok) {
                atomicExch(&bar->dead, 1);
                for (int s = 0; s < sh.nscn; ++s) atomicOr(&sh.scn[s].ctl->err, ERR_TIMEOUT);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Shared memory of the persistent kernel: the largest phase's, reused by
// every phase (each phase initialises what it reads).
constexpr size_t PERSIST_SMEM = sizeof(P2CSmem) > sizeof(P2SSmem) ? (sizeof(P2CSmem) > sizeof(G2PSmem) ? sizeof(P2CSmem) : sizeof(G2PSmem))
                                                                  : (sizeof(P2SSmem) > sizeof(G2PSmem) ? sizeof(P2SSmem) : sizeof(G2PSmem));

// Up to nsteps whole steps (K1 tile bookkeeping, K2 both P2G classes, K3 grid
// update, K4 G2P, K5 end of step) in one launch, the phases separated by
// grid_sync instead of kernel boundaries. The same phase bodies as the
// separate kernels, over the same work lists and in the same per-tile order,
// so a step gives the same bits either way. The launch ends early once no
// scenario has work (every one stopped at its frame, step budget or end).
__global__ void __launch_bounds__(NCELL, P2C_MIN_BLOCKS) k_persist(Shared sh, const double* __restrict__ z64, int nsteps, long long limit,
                                                                   GridBar* bar, const __grid_constant__ CUtensorMap dem_map) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // after a launch whose waits ran out, the tile bookkeeping of the step it
    // left is half done: no phase may run on it again
    if (*reinterpret_cast<volatile const int*>(&bar->dead)) return;
    for (int s = 0; s < nsteps; ++s) {
        prep_body(sh);
        if (!grid_sync(sh, bar, limit)) return;
        p2g_cell_body<false>(sh, 0, smem_raw, &dem_map);
        __syncthreads();  // the shared memory passes to the next phase
        p2g_sparse_body(sh, 1, smem_raw);
        if (!grid_sync(sh, bar, limit)) return;
        grid_body(sh);
        if (!grid_sync(sh, bar, limit)) return;
        g2p_body(sh, z64, *reinterpret_cast<G2PSmem*>(smem_raw));
        if (!grid_sync(sh, bar, limit)) return;
        if (blockIdx.x == 0) end_body(sh);
        if (!grid_sync(sh, bar, limit)) return;
        if (*reinterpret_cast<volatile const int*>(sh.work_pref + sh.nscn) == 0) break;  // the same value in every CTA
    }
}

// Particle z and vz at the current positions (for downloads between output
// frames, where the step loop does not keep them): vz = v . grad z of the
// containing cell, z from the quadratic stencil of FP64 terrain heights.
__global__ void k_refresh_vz_z(Shared sh, PBuf B, int Np, const double* __restrict__ z64) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < Np; q += gridDim.x * blockDim.x) {
        const int32_t cell = B.cell[q];
        const float2 f = B.f[q], v = B.v[q];
        const int i0 = cell_i(cell), j0 = cell_j(cell);
        float wx[3], wy[3], dwx[3], dwy[3];
        bspline3(f.x, wx, dwx);
        bspline3(f.y, wy, dwy);
        const float4 dm = sh.dem[(int64_t)(i0 + (f.x >= 1.f ? 1 : 0)) * sh.Ny + (j0 + (f.y >= 1.f ? 1 : 0))];
        double zp = 0.0;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) zp += (double)(wx[a] * wy[b]) * z64[(int64_t)(i0 + a) * sh.Ny + (j0 + b)];
        B.vz[q] = v.x * dm.x + v.y * dm.y;
        B.z[q] = (float)zp;
    }
}

}  // namespace k32
}  // namespace slab
