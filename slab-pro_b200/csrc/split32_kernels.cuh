// Kernels of the FP32 split-precision step loop (K1-K6), shared by the
// single-scenario path and the batched / served paths. One step is
//   k_begin  (1 CTA)   per-scenario dt / stop rules, work-list prefix
//   k_prep   (grid)    one thread per active tile: its 9 particle groups,
//                      its segment in the next buffer, grid-tile list
//   k_p2g    (grid)    one CTA per active tile: P2G partial sums
//   k_grid   (grid)    one CTA per grid tile: grid update + friction
//   k_g2p    (grid)    one CTA per active tile: G2P, advection, regrouping
// The CTAs stride over a flat list of work items of all scenarios, so one
// launch advances every running scenario by one step, each with its own dt
// and friction law.
#pragma once

#include "split32.cuh"

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

__device__ __forceinline__ int seq_to_index(int q, const TileDesc& D) {
    int d = 0;
    while (d < 8 && D.gpref[d + 1] <= q) ++d;
    return D.gstart[d] + (q - D.gpref[d]);
}

// copy a descriptor to shared memory (threads 0..23)
__device__ __forceinline__ void load_desc(const TileDesc* g, TileDesc* s) {
    if (threadIdx.x < (int)(sizeof(TileDesc) / 4)) reinterpret_cast<int*>(s)[threadIdx.x] = reinterpret_cast<const int*>(g)[threadIdx.x];
}

// ---------------------------------------------------------------- control

// K5 (first half): per scenario, Simulation::updateDt and the stop rules;
// then the prefix of active tiles over scenarios (the work list).
__global__ void k_begin(Shared sh, int t0_pass) {
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
            } else {
                ctl_begin(c, sh.Nx, sh.Ny);
            }
            if (c->active) {
                n->stepid += 1;
                n->act_count[(n->seq + 1) & 1] = 0;
                n->gt_count = 0;
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
        sh.done[0] = 0;
        sh.done[1] = 0;
    }
}

// K1 (bookkeeping half): one thread per active tile. Tile t's particles are
// group d of the 9 neighbour segments t - dir(d) of the current buffer; the
// descriptor records them, reserves the tile's segment in the next buffer
// and puts the 4 tiles owning its node window on the grid-tile list.
__global__ void __launch_bounds__(256) k_prep(Shared sh) {
    const int nwork = sh.work_pref[sh.nscn];
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < nwork; w += gridDim.x * blockDim.x) {
        int sid, loc;
        find_work(sh.work_pref, sh.nscn, w, sid, loc);
        const Scn& S = sh.scn[sid];
        SCnt* n = S.cnt;
        const int seq = n->seq, cur = seq & 1;
        const int t = S.act_list[cur][loc];
        const int ti = t / sh.TY, tj = t % sh.TY;
        TileDesc D;
        D.t = t;
        D.sid = sid;
        int st[9], en[9];
#pragma unroll
        for (int d = 0; d < 9; ++d) {
            const int si = ti - dir_i(d), sj = tj - dir_j(d);
            st[d] = en[d] = 0;
            if (si >= 0 && sj >= 0 && si < sh.TX && sj < sh.TY) {
                const int s = si * sh.TY + sj;
                if (S.grp_stamp[cur][s] == seq) {
                    st[d] = S.grp[cur][s * 10 + d];
                    en[d] = S.grp[cur][s * 10 + d + 1];
                }
            }
        }
        int acc = 0;
#pragma unroll
        for (int d = 0; d < 9; ++d) {
            D.gstart[d] = st[d];
            D.gpref[d] = acc;
            acc += en[d] - st[d];
        }
        D.gpref[9] = acc;
        D.total = acc;
        D.nxt_off = atomicAdd(&n->cursor, acc);
        D.pad_ = 0;
        S.slot_of[t] = w;
        const int stamp = n->stepid;
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                const int gi = ti + a, gj = tj + b;
                if (gi < sh.TX && gj < sh.TY) {
                    const int g = gi * sh.TY + gj;
                    if (atomicMax(&S.gt_stamp[g], stamp) < stamp) S.gt_list[atomicAdd(&n->gt_count, 1)] = g;
                }
            }
        sh.desc[w] = D;
    }
    // the last CTA builds the grid-tile work list prefix for k_grid
    __shared__ int s_last, s_tot;
    __shared__ int s_warp[33];
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = (atomicAdd(&sh.done[0], 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        int total = 0;
        for (int base = 0; base < sh.nscn; base += blockDim.x) {
            const int s = base + threadIdx.x;
            const int cnt = (s < sh.nscn && sh.scn[s].ctl->active) ? *(volatile int*)&sh.scn[s].cnt->gt_count : 0;
            const int ex = block_exclusive_scan(cnt, s_warp);
            if (s < sh.nscn) sh.grid_pref[s] = total + ex;
            if (threadIdx.x == blockDim.x - 1) s_tot = ex + cnt;
            __syncthreads();
            total += s_tot;
            __syncthreads();
        }
        if (threadIdx.x == 0) sh.grid_pref[sh.nscn] = total;
    }
}

// ------------------------------------------------------------------- P2G

struct P2GSmem {
    float node[NQ * TN * TN];
    float4 dem[(TILE + 1) * (TILE + 1)];
    int lc[CHUNK];
    float2 f[CHUNK];
    float2 v[CHUNK];
    float h[CHUNK];
    float m[CHUNK];
    float vz[CHUNK];
    short idx[CHUNK];
    int ccnt[NCELL];
    int ccur[NCELL];
    int warp[NCELL / 32 + 1];
    TileDesc d;
};

// K2: P2G of one tile (src/simulation.cpp:726-798) without atomics on the
// sums. Each thread owns one base cell of the tile and sums the
// contributions of that cell's particles to its 3x3 nodes in registers,
// visiting the particles in a fixed order (the tile's particle sequence,
// bucketed by cell in shared memory). The register blocks are combined into
// the shared (TILE+2)^2 node window along j with warp shuffles and along i in
// 3 conflict-free phases; the window is written as the tile's partial sums.
__global__ void __launch_bounds__(NCELL, 2) k_p2g(Shared sh) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    P2GSmem& sm = *reinterpret_cast<P2GSmem*>(smem_raw);
    const int tid = threadIdx.x;
    const int ci = tid / TILE, cj = tid % TILE;
    const int nwork = sh.work_pref[sh.nscn];
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        load_desc(sh.desc + w, &sm.d);
        __syncthreads();
        const Scn& S = sh.scn[sm.d.sid];
        const int t = sm.d.t;
        const int ti = t / sh.TY, tj = t % sh.TY;
        SCnt* n = S.cnt;
        const int cur = n->seq & 1;
        const bool outs = n->outs != 0;
        for (int k = tid; k < (TILE + 1) * (TILE + 1); k += NCELL) {
            const int i = ti * TILE + k / (TILE + 1), j = tj * TILE + k % (TILE + 1);
            sm.dem[k] = (i < sh.Nx && j < sh.Ny) ? sh.dem[(int64_t)i * sh.Ny + j] : make_float4(0.f, 0.f, 1.f, 0.f);
        }
        for (int k = tid; k < NQ * TN * TN; k += NCELL) sm.node[k] = 0.f;
        const int total = sm.d.total;
        const PBuf B = S.buf[cur];
        const float g = S.g, ood = S.ood;
        float acc[9][NQ];
#pragma unroll
        for (int a = 0; a < 9; ++a)
#pragma unroll
            for (int q = 0; q < NQ; ++q) acc[a][q] = 0.f;
        for (int c0 = 0; c0 < total; c0 += CHUNK) {
            const int nc = min(CHUNK, total - c0);
            sm.ccnt[tid] = 0;
            __syncthreads();
            for (int k = tid; k < nc; k += NCELL) {
                const int src = seq_to_index(c0 + k, sm.d);
                const int32_t cell = B.cell[src];
                int li = cell_i(cell) - ti * TILE, lj = cell_j(cell) - tj * TILE;
                if ((unsigned)li >= TILE || (unsigned)lj >= TILE) {
                    atomicOr(&S.ctl->err, ERR_MOVE);
                    li = min(max(li, 0), TILE - 1);
                    lj = min(max(lj, 0), TILE - 1);
                }
                const int lc = li * TILE + lj;
                sm.lc[k] = lc;
                sm.f[k] = B.f[src];
                sm.v[k] = B.v[src];
                sm.h[k] = B.h[src];
                sm.m[k] = B.m[src];
                sm.vz[k] = outs ? B.vz[src] : 0.f;
                atomicAdd(&sm.ccnt[lc], 1);
            }
            __syncthreads();
            const int my_cnt = sm.ccnt[tid];
            const int my_start = block_exclusive_scan(my_cnt, sm.warp);
            sm.ccur[tid] = my_start;
            __syncthreads();
            for (int k = tid; k < nc; k += NCELL) sm.idx[atomicAdd(&sm.ccur[sm.lc[k]], 1)] = (short)k;
            __syncthreads();
            // this cell's particles in sequence order (insertion sort of the
            // few indices the scatter above placed in arbitrary order)
            for (int a = 1; a < my_cnt; ++a) {
                const short key = sm.idx[my_start + a];
                int b = a - 1;
                while (b >= 0 && sm.idx[my_start + b] > key) {
                    sm.idx[my_start + b + 1] = sm.idx[my_start + b];
                    --b;
                }
                sm.idx[my_start + b + 1] = key;
            }
            for (int a = 0; a < my_cnt; ++a) {
                const int k = sm.idx[my_start + a];
                const float2 f = sm.f[k], v = sm.v[k];
                const float h = sm.h[k], m = sm.m[k];
                float wx[3], wy[3], dwx[3], dwy[3];
                bspline3(f.x, wx, dwx);
                bspline3(f.y, wy, dwy);
                // slope terms of the containing cell (src/complex_terrain.cpp:113-130)
                const float4 dm = sm.dem[(ci + (f.x >= 1.f ? 1 : 0)) * (TILE + 1) + (cj + (f.y >= 1.f ? 1 : 0))];
                // gravity along the slope and the depth-averaged pressure
                // sigma = -rho g cos^2 h / 2 with h A = m / rho
                // (src/simulation.cpp:744-756, 786-793)
                const float K = m * g * dm.z * dm.z;
                const float hh = 0.5f * h * ood;
                const float mvx = m * v.x, mvy = m * v.y, mh = m * h, mvz = m * sm.vz[k];
#pragma unroll
                for (int ia = 0; ia < 3; ++ia) {
#pragma unroll
                    for (int jb = 0; jb < 3; ++jb) {
                        const float wgt = wx[ia] * wy[jb];
                        if (wgt > 3e-3f) {  // the reference's weight cut-off (src/simulation.cpp:780)
                            float* A = acc[ia * 3 + jb];
                            A[0] += m * wgt;
                            A[1] += mvx * wgt;
                            A[2] += mvy * wgt;
                            A[3] += mh * wgt;
                            A[4] += K * (hh * dwx[ia] * wy[jb] - dm.x * wgt);
                            A[5] += K * (hh * dwy[jb] * wx[ia] - dm.y * wgt);
                            A[6] += mvz * wgt;
                        }
                    }
                }
            }
            __syncthreads();
        }
        // Combine: node (ci+a, nj) gets acc[a][0] of cell nj, acc[a][1] of
        // cell nj-1 and acc[a][2] of cell nj-2 (same row of the tile, i.e.
        // adjacent lanes), then rows are added in 3 phases a = 0, 1, 2.
#pragma unroll
        for (int ia = 0; ia < 3; ++ia) {
            float* row = sm.node + (ci + ia) * TN;
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                const float a0 = acc[ia * 3 + 0][q], a1 = acc[ia * 3 + 1][q], a2 = acc[ia * 3 + 2][q];
                const float s1 = __shfl_up_sync(0xffffffffu, a1, 1);
                const float s2 = __shfl_up_sync(0xffffffffu, a2, 2);
                const float s21 = __shfl_up_sync(0xffffffffu, a2, 1);
                float val = a0;
                if (cj >= 1) val += s1;
                if (cj >= 2) val += s2;
                row[q * TN * TN + cj] += val;
                if (cj == TILE - 1) {
                    row[q * TN * TN + TILE] += a1 + s21;  // cells 15 (b=1) and 14 (b=2)
                    row[q * TN * TN + TILE + 1] += a2;    // cell 15 (b=2)
                }
            }
            __syncthreads();
        }
        float* P = sh.part + (size_t)w * PART_STRIDE;
        for (int k = tid; k < PART_STRIDE; k += NCELL) P[k] = sm.node[k];
        __syncthreads();
    }
}

// ------------------------------------------------------------ grid update

// K3 + K6: computeGridVelocity (src/simulation.cpp:800-875) for the TILE^2
// nodes owned by one grid tile. A node's P2G sum is the partials of the
// tiles whose window covers it, added in a fixed order (own, -x, -y, -xy).
// h_max / v_max2 are updated in the node block; the FP64 grid mass sum is
// the conservation diagnostic.
__global__ void __launch_bounds__(NCELL) k_grid(Shared sh) {
    __shared__ int s_sid, s_loc, s_blk;
    __shared__ int s_slot[4];
    __shared__ double s_red[NCELL / 32];
    __shared__ unsigned s_act[NCELL / 32];
    const int tid = threadIdx.x;
    const int li = tid / TILE, lj = tid % TILE;
    const int nwork = sh.grid_pref[sh.nscn];
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        if (tid == 0) find_work(sh.grid_pref, sh.nscn, w, s_sid, s_loc);
        __syncthreads();
        const Scn& S = sh.scn[s_sid];
        SCnt* n = S.cnt;
        Ctl* c = S.ctl;
        const int gt = S.gt_list[s_loc];
        const int gi = gt / sh.TY, gj = gt % sh.TY;
        if (tid < 4) {
            // contributor k: tile (gi - (k>>1), gj - (k&1)); slot if active this step
            const int ti_ = gi - (tid >> 1), tj_ = gj - (tid & 1);
            int slot = -1;
            if (ti_ >= 0 && tj_ >= 0) {
                const int tt = ti_ * sh.TY + tj_;
                if (S.act_stamp[tt] == n->seq) slot = S.slot_of[tt];
            }
            s_slot[tid] = slot;
        } else if (tid == 32) {
            int blk = S.blk_of[gt];
            if (blk < 0) {
                blk = atomicAdd(sh.blk_count, 1);
                if (blk >= sh.blk_cap) {
                    atomicOr(&c->err, ERR_CAPACITY);
                    blk = -1;
                } else {
                    S.blk_of[gt] = blk;
                    sh.blk_owner[blk] = s_sid;
                }
            }
            if (blk >= 0) sh.blk_stamp[blk] = n->stepid;
            s_blk = blk;
        }
        __syncthreads();
        const int blk = s_blk;
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
            add(s_slot[0], li, lj);
            if (li < 2) add(s_slot[2], li + TILE, lj);
            if (lj < 2) add(s_slot[1], li, lj + TILE);
            if (li < 2 && lj < 2) add(s_slot[3], li + TILE, lj + TILE);
            const int i = gi * TILE + li, j = gj * TILE + lj;
            const size_t bn = (size_t)blk * NCELL + tid;
            float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
            float hn = 0.f, vzn = 0.f;
            const float mi = q[0];
            if (mi > 1e-6f && i < sh.Nx && j < sh.Ny) {
                const float vox = q[1] / mi, voy = q[2] / mi;
                vzn = q[6] / mi;
                hn = q[3] / mi;
                const float dt = (float)c->dt;
                const float vtx = vox + dt * (q[4] / mi), vty = voy + dt * (q[5] / mi);
                const float vsq = vtx * vtx + vty * vty;
                float nvx = 0.f, nvy = 0.f;
                if (vsq > 1e-16f) {
                    const float4 dm = sh.dem[(int64_t)i * sh.Ny + j];
                    const float ct = dm.z;
                    const float vz = vtx * dm.x + vty * dm.y;
                    const float v3sq = vsq + vz * vz;
                    const float v3 = sqrtf(v3sq);
                    float af;
                    if (S.fric == SLAB_COULOMB) {
                        af = S.mu_c * S.g * ct;
                    } else if (S.fric == SLAB_VOELLMY) {
                        af = S.mu_v * S.g * ct + S.g * v3sq / (S.xi * hn * ct);
                    } else {
                        const float I = 5.f * S.d * v3 / (2.f * hn * ct * ct * sqrtf(S.g * hn * S.phi));
                        const float muI = S.mu1 + (S.mu2 - S.mu1) / (1.f + S.I0 / I);
                        af = muI * S.g * ct;
                    }
                    const float dv = dt * af;
                    if (dv < v3) {
                        const float fct = 1.f - dv / v3;
                        nvx = vtx * fct;
                        nvy = vty * fct;
                    }
                }
                out = make_float4(nvx, nvy, nvx - vox, nvy - voy);
                sh.hmax[bn] = fmaxf(sh.hmax[bn], hn);
                sh.vmax2[bn] = fmaxf(sh.vmax2[bn], nvx * nvx + nvy * nvy);
                mloc = (double)mi;
            }
            sh.nv[bn] = out;
            if (n->outs) {
                sh.oh[bn] = hn;
                sh.om[bn] = (i < sh.Nx && j < sh.Ny) ? mi : 0.f;
                sh.ovz[bn] = vzn;
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
            if (sum != 0.0) atomicAdd(&n->grid_mass, sum);
            if (na) atomicAdd(&c->node_steps, (unsigned long long)na);
        }
        __syncthreads();
    }
}

// -------------------------------------------------------------------- G2P

// New base cell and offset of a particle after advection with the PIC
// velocity of the 3x3 nodes around it. One out-of-line function serves both
// passes of k_g2p, so both classify every particle identically.
__device__ __noinline__ void advect(const float4* s_nv, int ci, int cj, int32_t cell, float2 f, float dt_ood, int* ib, int* jb,
                                   float2* fnew, float2* pic) {
    float wx[3], wy[3], dwx[3], dwy[3];
    bspline3(f.x, wx, dwx);
    bspline3(f.y, wy, dwy);
    float picx = 0.f, picy = 0.f;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const float w = wx[a] * wy[b];
            const float4 nv = s_nv[(ci + a) * TN + (cj + b)];
            picx += nv.x * w;
            picy += nv.y * w;
        }
    const float ux = f.x + dt_ood * picx, uy = f.y + dt_ood * picy;
    const int ki = (int)floorf(ux - 0.5f), kj = (int)floorf(uy - 0.5f);
    *ib = cell_i(cell) + ki;
    *jb = cell_j(cell) + kj;
    *fnew = make_float2(ux - (float)ki, uy - (float)kj);
    *pic = make_float2(picx, picy);
}

__device__ __forceinline__ int dir_of(int ib, int jb, int ti, int tj) {
    int di = (ib >= 0 ? ib / TILE : -1) - ti, dj = (jb >= 0 ? jb / TILE : -1) - tj;
    if (di < -1 || di > 1 || dj < -1 || dj > 1) return -1;
    return (di + 1) * 3 + (dj + 1);
}

struct G2PSmem {
    float4 nv[TN * TN];
    float4 dem[(TILE + 1) * (TILE + 1)];
    int dcnt[9];
    int dpref[10];
    int wtot[NCELL / 32][9];
    int run[9];
    int blk4[4];
    TileDesc d;
    double red[5][NCELL / 32];
};

// K4: G2P (src/simulation.cpp:877-940) of one tile: FLIP/PIC blend,
// advection, depth update, then the particle is written to the next buffer
// in the group of the tile it moved to. Pass 1 counts the groups, pass 2
// writes each particle at its stable rank. The block max of |v|^2 and the
// particle bounding box feed the next step's dt and remesh box (K5).
__global__ void __launch_bounds__(NCELL, 2) k_g2p(Shared sh, const double* __restrict__ z64) {
    __shared__ G2PSmem sm;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nwork = sh.work_pref[sh.nscn];
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        load_desc(sh.desc + w, &sm.d);
        __syncthreads();
        const int sid = sm.d.sid;
        const Scn& S = sh.scn[sid];
        SCnt* n = S.cnt;
        Ctl* c = S.ctl;
        const int seq = n->seq, cur = seq & 1, nxt = cur ^ 1;
        const int t = sm.d.t;
        const int ti = t / sh.TY, tj = t % sh.TY;
        const bool outs = n->outs != 0;
        const bool need_vz = outs || n->vz_next;
        if (tid < 4) {
            const int gi = ti + (tid >> 1), gj = tj + (tid & 1);
            sm.blk4[tid] = (gi < sh.TX && gj < sh.TY) ? S.blk_of[gi * sh.TY + gj] : -1;
        }
        if (tid >= 32 && tid < 41) sm.dcnt[tid - 32] = 0;
        __syncthreads();
        for (int k = tid; k < TN * TN; k += NCELL) {
            const int a = k / TN, b = k % TN;
            const int i = ti * TILE + a, j = tj * TILE + b;
            float4 val = make_float4(0.f, 0.f, 0.f, 0.f);
            if (i < sh.Nx && j < sh.Ny) {
                const int blk = sm.blk4[(a >= TILE ? 2 : 0) + (b >= TILE ? 1 : 0)];
                if (blk >= 0) val = sh.nv[(size_t)blk * NCELL + (a % TILE) * TILE + (b % TILE)];
            }
            sm.nv[k] = val;
        }
        if (need_vz) {
            for (int k = tid; k < (TILE + 1) * (TILE + 1); k += NCELL) {
                const int i = ti * TILE + k / (TILE + 1), j = tj * TILE + k % (TILE + 1);
                sm.dem[k] = (i < sh.Nx && j < sh.Ny) ? sh.dem[(int64_t)i * sh.Ny + j] : make_float4(0.f, 0.f, 1.f, 0.f);
            }
        }
        __syncthreads();
        const int total = sm.d.total;
        const PBuf B = S.buf[cur];
        const PBuf O = S.buf[nxt];
        const float dt = (float)c->dt;
        const float dt_ood = dt * S.ood;
        const double dx = c->dx;
        // pass 1: count the particles per destination group
        for (int q = tid; q < total; q += NCELL) {
            const int src = seq_to_index(q, sm.d);
            const int32_t cell = B.cell[src];
            const float2 f = B.f[src];
            const int ci = min(max(cell_i(cell) - ti * TILE, 0), TILE - 1);
            const int cj = min(max(cell_j(cell) - tj * TILE, 0), TILE - 1);
            int ib, jb;
            float2 fn, pic;
            advect(sm.nv, ci, cj, cell, f, dt_ood, &ib, &jb, &fn, &pic);
            const int d = dir_of(ib, jb, ti, tj);
            atomicAdd(&sm.dcnt[d < 0 ? 4 : d], 1);
        }
        __syncthreads();
        if (tid < 10) {
            int acc = 0;
            for (int d = 0; d < tid; ++d) acc += sm.dcnt[d];
            sm.dpref[tid] = acc;
            S.grp[nxt][t * 10 + tid] = sm.d.nxt_off + acc;
            if (tid < 9) {
                sm.run[tid] = 0;
                if (sm.dcnt[tid]) {
                    const int tt = (ti + dir_i(tid)) * sh.TY + (tj + dir_j(tid));
                    if (atomicMax(&S.act_stamp[tt], seq + 1) < seq + 1) {
                        const int k = atomicAdd(&n->act_count[nxt], 1);
                        if (k < S.act_cap) S.act_list[nxt][k] = tt;
                        else atomicOr(&c->err, ERR_CAPACITY);
                    }
                }
            } else {
                S.grp_stamp[nxt][t] = seq + 1;
            }
        }
        __syncthreads();
        // pass 2: full update, stable write into the destination groups
        double mnx = INFINITY, mxx = 0.0, mny = INFINITY, mxy = 0.0, vv = 0.0;
        for (int r0 = 0; r0 < total; r0 += NCELL) {
            const int q = r0 + tid;
            const bool valid = q < total;
            int d = 4, ib = 0, jb = 0;
            float2 fn = make_float2(1.f, 1.f), vn = make_float2(0.f, 0.f);
            float hn = 0.f, m = 0.f, vzp = 0.f;
            double zp = 0.0;
            int32_t pid = 0;
            if (valid) {
                const int src = seq_to_index(q, sm.d);
                const int32_t cell = B.cell[src];
                const float2 f = B.f[src];
                const float2 v = B.v[src];
                const float h = B.h[src];
                m = B.m[src];
                pid = B.id[src];
                const int ci = min(max(cell_i(cell) - ti * TILE, 0), TILE - 1);
                const int cj = min(max(cell_j(cell) - tj * TILE, 0), TILE - 1);
                float2 pic;
                advect(sm.nv, ci, cj, cell, f, dt_ood, &ib, &jb, &fn, &pic);
                float wx[3], wy[3], dwx[3], dwy[3];
                bspline3(f.x, wx, dwx);
                bspline3(f.y, wy, dwy);
                float flx = 0.f, fly = 0.f, div = 0.f;
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int b = 0; b < 3; ++b) {
                        const float wgt = wx[a] * wy[b];
                        const float4 nv = sm.nv[(ci + a) * TN + (cj + b)];
                        flx += nv.z * wgt;
                        fly += nv.w * wgt;
                        div += (dwx[a] * wy[b]) * nv.x + (dwy[b] * wx[a]) * nv.y;
                    }
                div *= S.ood;
                const float fr = S.fr;
                vn = make_float2(fr * (v.x + flx) + (1.f - fr) * pic.x, fr * (v.y + fly) + (1.f - fr) * pic.y);
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
                d = dir_of(ib, jb, ti, tj);
                if (d < 0) {
                    atomicOr(&c->err, ERR_MOVE);
                    d = 4;
                }
                if (ib < 0 || jb < 0 || ib + 2 > sh.Nx - 1 || jb + 2 > sh.Ny - 1) {
                    atomicOr(&c->err, ERR_DOMAIN);
                    ib = min(max(ib, 0), sh.Nx - 3);
                    jb = min(max(jb, 0), sh.Ny - 3);
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
            int rank = 0;
#pragma unroll
            for (int dd = 0; dd < 9; ++dd) {
                const unsigned msk = __ballot_sync(0xffffffffu, valid && d == dd);
                if (lane == 0) sm.wtot[warp][dd] = __popc(msk);
                if (valid && d == dd) rank = __popc(msk & ((1u << lane) - 1u));
            }
            __syncthreads();
            if (tid < 9) {
                int run = sm.run[tid];
                for (int wp = 0; wp < NCELL / 32; ++wp) {
                    const int tmp = sm.wtot[wp][tid];
                    sm.wtot[wp][tid] = run;
                    run += tmp;
                }
                sm.run[tid] = run;
            }
            __syncthreads();
            if (valid) {
                const int pos = sm.d.nxt_off + sm.dpref[d] + sm.wtot[warp][d] + rank;
                O.cell[pos] = pack_cell(ib, jb);
                O.f[pos] = fn;
                O.v[pos] = vn;
                O.h[pos] = hn;
                O.m[pos] = m;
                O.id[pos] = pid;
                if (need_vz) O.vz[pos] = vzp;
                if (outs) O.z[pos] = (float)zp;
            }
            __syncthreads();
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
    }
    // the last CTA closes the step of every running scenario
    __shared__ int s_last;
    if (tid == 0) {
        __threadfence();
        s_last = (atomicAdd(&sh.done[1], 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        for (int s = tid; s < sh.nscn; s += blockDim.x) {
            const Scn& S = sh.scn[s];
            Ctl* c = S.ctl;
            if (!c->active) continue;
            SCnt* n = S.cnt;
            if (*(volatile int*)&n->cursor != S.Np) atomicOr(&c->err, ERR_CAPACITY);
            ctl_end(c);
            n->seq += 1;
            n->vz_valid = n->outs;
        }
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
