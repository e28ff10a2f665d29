// Host object that owns the device state of one or many FP32 split-precision
// scenarios on a shared terrain and launches their steps together.
#pragma once

#include <cuda.h>

#include <string>

#include <deque>
#include <memory>
#include <vector>

#include "engine.hpp"
#include "split32.cuh"

namespace slab {

class Engine32 {
  public:
    struct Store {
        int Np = 0;
        int act_cap = 0;
        int Np_alloc = 0;   // particle buffer length
        int act_alloc = 0;  // tile list length
        Ctl* ctl = nullptr;
        Ctl* h_ctl = nullptr;
        dptr<int32_t> cell[2], id[2], grp[2], act_list[2];
        dptr<float2> f[2], v[2];
        dptr<float> h[2], m[2], vz[2], z[2];
        dptr<int32_t> act_stamp, slot_of, nxt_off, gt_stamp, blk_of;
        SCnt* cnt = nullptr;  // in the engine's counter array
    };

    Engine32(const Terrain& t, cudaStream_t s, int max_scenarios, int64_t blk_cap, bool batch = false);
    ~Engine32();

    // want_slot >= 0: use that free slot (or the next unused one)
    int add_scenario(const slab_params& p, Ctl* ctl, Ctl* h_ctl, int Np, const double* x, const double* v, const double* vz,
                     const double* h, const double* m, const double* z, int want_slot = -1);
    void launch_begin(int t0);
    void launch_t0();
    void launch_step();
    void launch_kernel(int k, const Shared& sh);
    void launch_p2g(const Shared& sh);
    void launch_p2g_cell(const Shared& sh, int cls);
    CUtensorMap dem_map;   // the FP32 terrain as [Nx][4 Ny] floats, 9 x 9-node boxes (the cell P2G's terrain window)
    bool p2g_tma = false;  // k_p2g_cell<true>: the next tile's loads staged by TMA bulk copies (SLAB_P2G_TMA=1)
    // persistent steps: a chunk of steps as one cooperative launch of k_persist
    // (SLAB_PERSIST=1 or set_persistent); its grid waits give up after
    // persist_limit clock cycles (ERR_TIMEOUT)
    bool persist = false;
    long long persist_limit = 4000000000ll;
    int grid_persist = 0;
    dptr<unsigned> d_bar;  // k32::GridBar
    bool dead = false;     // a persistent launch gave up: no further steps
    void set_persistent(bool on, long long limit_cycles);
    void launch_persistent(int chunk);
    void arm(int64_t steps_left, int stop_at_frame);
    int acc_mode = 5;  // P2G scheme (k32::ACC_*): dense tiles cell-sorted, sparse tiles fixed point
    int split_min = 3 * NCELL / 4;  // ACC_MIXED: tiles with more particles take the cell-sorted P2G (measured)
    void enqueue_steps(int chunk);
    PhaseTimer timer;
    SCnt counters(int sid);
    // grow per-scenario tile lists and the node-block pool when half full;
    // returns true if anything was reallocated
    bool check_capacity();
    void grow_blocks(int cap);
    // free a finished scenario's slot: its memory, its node blocks (back to
    // the pool, zeroed) and its control block (replaced by empty_ctl)
    void retire(int sid, const Ctl& empty_ctl);
    // node box covered by the scenario's blocks; box[1] < box[0] if none
    void box_of_blocks(int sid, int box[4]);
    void download_max_box(int sid, const int box[4], double* hmax, double* vmax2);
    void download_particles(int sid, double* x, double* v, double* vz, double* h, double* A, double* m, double* z, double rho);
    void download_grid(int sid, slab_grid_view* gv);
    void download_max(int sid, double* hmax, double* vmax2);
    void conservation(int sid, double out[4], double rho);
    void moments(int sid, double out[6]);
    // the current frame in the output files' float32 layouts (slab_frame_capture)
    void pack_frame(int sid, float* d_part, float* d_grid, const int32_t box[4], double rho);
    dptr<double> d_mom;  // moment partials and result (moments.cuh)
    Shared shared() const;

    const Terrain& T;
    cudaStream_t st;
    int max_scn;
    bool batch = false;
    int nscn = 0;
    int TX = 0, TY = 0, ntiles = 0;
    int blk_cap = 0;
    int64_t pending_blocks = 0;  // node blocks of scenarios added since the last t=0 pass (an estimate)
    int grid_p2g = 0, grid_p2g_cell = 0, grid_p2g_hilo = 0, grid_p2g_sparse = 0, grid_g2p = 0, grid_grid = 0, grid_prep = 0;

    // Launch-shape tuner of the step's five work kernels (k_prep, k_p2g_cell,
    // k_p2g_sparse, k_grid, k_g2p). Each CTA of these kernels takes a
    // contiguous slice of a device-built work list and every work item is
    // computed by one CTA alone, so the grid size changes which CTA computes a
    // tile, never a value: all candidates give bitwise the same results. The
    // tuner times the candidates on live steps, interleaved (schedule step s
    // runs candidate s mod NC, so a workload that changes during the schedule
    // weighs on all candidates alike), and keeps per kernel the fastest. It
    // tunes on the first steps, again after 4x as many steps as at the last
    // pick, and when the active tile count has halved or doubled.
    struct Tuner {
        static constexpr int NK = 5, NC = 5, ROUNDS = 3, NSTEP = NC * ROUNDS;
        static constexpr int FACTOR4[NC] = {1, 2, 4, 8, 16};  // grid = occupancy grid * FACTOR4[c] / 4
        bool enabled = true;
        int state = 0;         // 0: shapes fixed, 1: measuring, 2: measured, events not read yet
        int done = 0;          // schedule steps launched
        int64_t steps = 0;     // steps enqueued
        int64_t next = 0;      // step count at which the next schedule starts
        int64_t active = 0;    // active tiles seen by the last capacity check
        int64_t active_at = 0; // active tiles when the last schedule started
        int base[NK] = {};     // occupancy-derived grids
        int pick[NK] = {2, 2, 2, 2, 2};
        int fixed[NK] = {};    // > 0: grid set by the caller, not tuned
        int tunes = 0;
        std::string key;       // a single scenario's workload size: picks shared by later contexts of the same size
        bool from_cache = false;
        std::vector<cudaEvent_t> ev;  // NK + 2 per schedule step
        ~Tuner() {
            for (auto e : ev) cudaEventDestroy(e);
        }
    } tune;
    int tuned_grid(int k, int c) const;
    void apply_shapes(const int* c);
    void tune_pick();
    void launch_step_timed(const Shared& sh, cudaEvent_t* e);
    // the five work kernels' grid sizes now in use
    void launch_shapes(int out[5]) const;
    // grids[k] > 0 fixes kernel k's grid (NULL: none fixed); tune_on: the tuner runs
    void fix_shapes(const int32_t* grids, bool tune_on);
    void tune_key_for(int Np);  // single scenario: picks of an earlier context of the same size, if any
    int work_cap = 0;
    int64_t work_cap_total = 0;
    void ensure_work_cap(int64_t need);
    int64_t nlaunch = 0;
    std::vector<std::unique_ptr<Store>> slots;  // scenario slots; empty after retire
    std::vector<std::unique_ptr<Store>> spare;  // a retired slot's arrays, for its next scenario
    dptr<int32_t> d_collect;                    // [ntiles + 8]: node blocks of one scenario, count and box
    dptr<float> d_gather;                       // node-field downloads
    size_t gather_cap = 0;
    dptr<const float*> d_gather_fp;
    Scratch scratch;                            // transient buffers of uploads (binning) and particle downloads
    dptr<int32_t> d_unpack_bad;                 // flag: a particle id out of range
    // node blocks of scenario sid: their ids into d_collect[8...], count and
    // tile box {ti0, ti1, tj0, tj1} to the host; returns the count
    int collect_blocks(int sid, int tbox[4]);
    std::vector<int> free_slots;
    std::vector<Scn> host_scn;

  private:
    std::vector<float> gather_nodes(int sid, int stepid, int i0, int j0, int nI, int nJ, const std::vector<const float*>& fields,
                                    bool with_v);
    dptr<float4> d_nv;
    dptr<float> d_hmax, d_vmax2, d_oh, d_om, d_ovz, d_oFx, d_oFy;
    dptr<int32_t> d_blk_stamp, d_blk_owner, d_misc, d_work_pref, d_gflat, d_wlist, d_free_blocks;
    dptr<Scn> d_scn;
    dptr<SCnt> d_cnt;
    std::vector<SCnt> h_cnt;
    dptr<TileDesc> d_desc;
    dptr<float> d_part;
    StepGraphs graphs;
    int graph_nscn = 0;
};

}  // namespace slab
