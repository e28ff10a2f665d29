/* slab_gpu.h -- C ABI of libslab_gpu.so, the B200 (sm_100a) engine for the
 * Slab-Pro depth-averaged material point method (MPM) time step.
 *
 * The reference (ALMO-SLF-ETH/Slab-Pro) has no plugin or FFI interface: its
 * boundary is the C++ class Simulation<T,TV2> (src/simulation.hpp:27-354),
 * whose simulate() (src/simulation.cpp:484-522) runs the step loop on the
 * host. This header is the interface that loop is replaced by. Each entry
 * point below names the reference code it stands in for. The C++ class in
 * slab-pro_b200/host/simulation.hpp keeps the reference's public Simulation
 * API and calls these functions from its simulate().
 *
 * Conventions
 *  - Plain C types only; every pointer argument is a host pointer unless the
 *    name says otherwise. The caller owns host buffers, a context owns its
 *    device memory.
 *  - Arrays follow the reference layouts (src/data_arrays.hpp:22-98):
 *    particle positions and velocities are interleaved (x0,y0,x1,y1,...) like
 *    std::vector<Eigen::Vector2d>; scalar particle fields are separate arrays;
 *    grid/terrain fields are flattened i*Ny + j (src/tools.hpp:172-174), with
 *    node (i,j) at (i*dx, j*dx).
 *  - Every function returns a slab_status. On error, slab_last_error() gives a
 *    message. The C++ wrapper rethrows non-OK codes as std::runtime_error,
 *    matching how the reference reports errors (src/main.cpp:52-55).
 *  - One context per host thread; contexts are not internally locked.
 */
#ifndef SLAB_GPU_H
#define SLAB_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum slab_status {
    SLAB_OK = 0,
    SLAB_E_ARG = 1,       /* invalid argument or size */
    SLAB_E_CUDA = 2,      /* CUDA runtime error (message has details) */
    SLAB_E_OOM = 3,       /* device allocation failed / capacity exceeded */
    SLAB_E_DOMAIN = 4,    /* a particle's 3x3 stencil left the terrain */
    SLAB_E_NONFINITE = 5, /* NaN/Inf in particle or grid state */
    SLAB_E_TIMEOUT = 6,   /* a bounded device-side wait gave up */
    SLAB_E_STATE = 7,     /* call out of order (e.g. advance before upload) */
    SLAB_E_NOTFOUND = 8   /* unknown scenario / request id */
} slab_status;

/* Basal friction laws, src/tools.hpp:37,62-84 */
typedef enum slab_friction_type { SLAB_COULOMB = 0, SLAB_VOELLMY = 1, SLAB_MU_I = 2 } slab_friction_type;

/* Arithmetic of the step loop.
 *  FP64_PLAIN: state and arithmetic in FP64, particles in upload order,
 *              atomicAdd(double) P2G scatter. The drop-in twin of the
 *              reference loop and the comparison baseline.
 *  FP32_SPLIT: positions as int32 cell index + FP32 in-cell offset, FP32
 *              particle/grid state, deterministic atomic-free P2G over
 *              cell-sorted particles in sparse 8x8-cell tiles. FP64 only for
 *              terrain metric terms, conservation sums, time and dt. */
typedef enum slab_precision { SLAB_FP64_PLAIN = 0, SLAB_FP32_SPLIT = 1 } slab_precision;

/* Friction parameters, src/tools.hpp:62-84 (struct Friction). */
typedef struct slab_friction {
    int32_t type; /* slab_friction_type */
    int32_t pad_;
    double coulomb_mu;
    double voellmy_mu, voellmy_xi;
    double mu_1, mu_2, I0, d, phi;
} slab_friction;

/* Simulation parameters read by Simulation::loadFromJSON
 * (src/simulation.cpp:118-208), plus the engine's precision. */
typedef struct slab_params {
    double gravity, rho;
    double C_cfl, dt_max, flip_ratio;
    double output_dt, total_time;
    slab_friction friction;
    int32_t precision; /* slab_precision */
    int32_t pad_;
} slab_params;

/* The terrain Grid of the reference (src/data_arrays.hpp:49-93,
 * src/complex_terrain.cpp:31-65): Nx x Ny nodes at spacing dx; the origin
 * offsets only matter for georeferenced output. */
typedef struct slab_terrain_desc {
    int32_t Nx, Ny;
    double dx;
    double xllcorner, yllcorner;
} slab_terrain_desc;

/* The remeshed grid the reference writes at every frame
 * (src/simulation.cpp:584-642, src/save_function.cpp:96-226), with the
 * members of class Grid (src/data_arrays.hpp:71-84) as computeGridVelocity
 * leaves them (src/simulation.cpp:800-875). The caller sets the pointers
 * (capacity given in cap_nodes; any pointer may be NULL); the call fills Nx,
 * Ny, i_off, j_off and the arrays (flattened i*Ny + j over the Nx x Ny box).
 * Every 2-vector field is interleaved (x, y). */
typedef struct slab_grid_view {
    int32_t Nx, Ny, i_off, j_off;
    int64_t cap_nodes;
    double* h;     /* Grid::h, normalised by the node mass */
    double* mass;  /* Grid::mass */
    double* v;     /* Grid::v after friction */
    double* vz;    /* Grid::vz */
    double* flip;  /* Grid::flip = v - v_old (zero where mass <= 1e-6) */
    double* F;     /* Grid::F, the P2G force sum */
    double* a;     /* Grid::a = F / mass (zero where mass <= 1e-6) */
} slab_grid_view;

typedef struct slab_ctx slab_ctx;

/* Create a context on the current CUDA device over terrain z[i*Ny+j].
 * Computes the terrain metric terms once, in FP64
 * (Simulation::terrainGradients / terrainTheta, src/complex_terrain.cpp:84-111)
 * and zeroes h_max / v_max2 (src/simulation.cpp:255-256). */
slab_status slab_create(const slab_terrain_desc* terrain, const double* z, slab_ctx** out);

/* Set the physical/numerical parameters (members filled by
 * Simulation::loadFromJSON, src/simulation.cpp:118-208). Must precede
 * slab_upload_particles. */
slab_status slab_set_params(slab_ctx* ctx, const slab_params* params);

/* Use this CUDA stream (a cudaStream_t) for every later call; NULL = the
 * context's own stream. */
slab_status slab_set_stream(slab_ctx* ctx, void* cuda_stream);

/* A release area of Simulation::initializeParticles (src/simulation.cpp:
 * 259-476) with UNIFORM 2x2 sampling: a RECTANGLE (a = Lx, b = Ly) or an
 * ELLIPSE (a = rx, b = ry) around (cx, cy), rotated by rotation_deg, of
 * uniform release height h0. Coordinates are relative to the terrain's
 * lower-left node, as the reference's release shapes are. */
enum { SLAB_RELEASE_RECTANGLE = 0, SLAB_RELEASE_ELLIPSE = 1 };
typedef struct slab_release {
    int32_t type; /* SLAB_RELEASE_* */
    int32_t pad_;
    double cx, cy;
    double a, b;
    double rotation_deg;
    double h0;
} slab_release;

/* Build the release's particles on the device -- the reference's setup
 * arithmetic, so the particles equal the reference's bit for bit: the
 * snapped bounding box, the 2x2 samples per cell filtered by the shape,
 * A = V / sum(h), mass = rho h A, z from the 4x4 stencil of terrain heights --
 * and upload them like slab_upload_particles (v = vz = 0). Np_out: the
 * particle count. SLAB_E_DOMAIN if the release reaches the terrain edge. */
slab_status slab_upload_release(slab_ctx* ctx, const slab_release* release, int32_t* Np_out);

/* Upload the particle set built by Simulation::initializeParticles
 * (src/simulation.cpp:259-476) -- the arrays of class Particles
 * (src/data_arrays.hpp:22-47). theta is derived on the device. Resets time,
 * dt and frame to zero. */
slab_status slab_upload_particles(slab_ctx* ctx, int32_t Np, const double* x_xy, const double* v_xy, const double* vz, const double* h,
                                  const double* A, const double* mass, const double* z);

/* simulate()'s t=0 pass (src/simulation.cpp:493-495): remesh, P2G and the
 * grid update with dt = 0, which normalises the grid fields for frame 0 and
 * seeds h_max. */
slab_status slab_initial_pass(slab_ctx* ctx);

/* Run iterations of simulate()'s loop (src/simulation.cpp:500-510, each one
 * Simulation::advanceStep, src/simulation.cpp:524-563, then time += dt) until
 * the next output frame is reached or time >= total_time. time and dt are
 * computed on the device exactly as Simulation::updateDt
 * (src/simulation.cpp:565-582), including the snap onto the frame time.
 * Outputs (any may be NULL): time after the last step, frame counter, and the
 * number of steps taken. */
slab_status slab_advance_to_frame(slab_ctx* ctx, double* time_out, int32_t* frame_out, int64_t* steps_out);

/* Run up to nsteps iterations of the same loop without stopping at frames
 * (frames still snap dt and bump the frame counter); stops early at
 * total_time. For benchmarks and tests. */
slab_status slab_advance_steps(slab_ctx* ctx, int64_t nsteps, int64_t* steps_out);

/* Enqueue nsteps iterations like slab_advance_steps on the context's stream
 * and return without waiting. The work and any device error are observed by
 * the next synchronising call (slab_synchronize or any download). */
slab_status slab_advance_steps_async(slab_ctx* ctx, int64_t nsteps);

/* Wait for the context's stream and report device-side errors. */
slab_status slab_synchronize(slab_ctx* ctx);

/* Copy the particle state back in the upload order (the reference reorders
 * particles every 50 steps, src/simulation.cpp:540; the engine keeps stable
 * ids instead). Any pointer may be NULL. A = mass/(h*rho) as in G2P
 * (src/simulation.cpp:938). z and vz are the values of the last step's G2P. */
slab_status slab_download_particles(slab_ctx* ctx, double* x_xy, double* v_xy, double* vz, double* h, double* A, double* mass, double* z);

/* The grid fields of the last step over the reference's remeshed bounding
 * box (src/simulation.cpp:603-612). With all four field pointers NULL only
 * the box (Nx, Ny, i_off, j_off) is filled in, to size the buffers. */
slab_status slab_download_grid(slab_ctx* ctx, slab_grid_view* view);

/* ---- output frames without stopping the step loop ----------------------
 * The reference writes particles_frame_N.ply and rasters_frame_N.tif at every
 * output frame from the host loop (src/simulation.cpp:496-497, 504-509;
 * src/save_function.cpp:36-226). Here a frame is packed on the device into
 * the files' own float32 layouts, copied to pinned host memory on a separate
 * copy stream while the next frame's steps run, and handed to the caller's
 * writer. Two slots: a capture into a slot first waits for that slot's
 * previous copy, and the caller must be done reading a slot's view before
 * capturing into it again. */
typedef struct slab_frame {
    int32_t frame;     /* output frame counter (Simulation::frame) */
    int32_t Np;
    double time;
    /* Np vertices of 8 float32: x y vx vy vz z h A, in upload order -- the
     * vertex layout of particles_frame_N.ply (src/save_function.cpp:44-75) */
    const float* particles;
    /* the frame's remeshed grid box (as slab_download_grid) and its 6 float32
     * bands h, |v|, m, vx, vy, vz of Nx*Ny values each in GeoTIFF order: row
     * 0 is the north edge (j = Ny - 1), x fastest; all bands -9999 where
     * h == 0 (src/save_function.cpp:96-226) */
    int32_t Nx, Ny, i_off, j_off;
    const float* grid;
} slab_frame;

/* Pack the current state (after slab_initial_pass or an advance call that
 * ended on a frame) into slot (0 or 1) and start its copy to the host; returns
 * without waiting for the copy. */
slab_status slab_frame_capture(slab_ctx* ctx, int32_t slot);
/* Wait for the slot's copy and fill *out; the pointers stay valid until the
 * slot is captured again or the context is destroyed. */
slab_status slab_frame_wait(slab_ctx* ctx, int32_t slot, slab_frame* out);

/* Full-terrain maxima (Grid::h_max, Grid::v_max2), as written by
 * Simulation::saveMaxData (src/save_function.cpp:228-291). Nx*Ny each. */
slab_status slab_download_max(slab_ctx* ctx, double* h_max, double* v_max2);

/* Diagnostics, all FP64: out[0] = total particle mass, out[1] = total grid
 * mass of the last step, out[2..3] = particle momentum (x, y). */
slab_status slab_conservation(slab_ctx* ctx, double out[4]);

/* Particle moments after the last step, all FP64 and summed on the device in
 * a fixed order: out[0] = total mass, out[1..2] = centre of mass (x, y),
 * out[3..4] = momentum (x, y), out[5] = kinetic energy sum m |v|^2 / 2. The
 * centre of mass frame by frame is the trajectory an FP32 run is compared
 * with an FP64 run on; the reference prints only the total volume
 * (src/simulation.cpp:473-475). */
slab_status slab_moments(slab_ctx* ctx, double out[6]);

/* time, dt, frame and steps so far (Simulation members time, dt, frame). */
slab_status slab_get_state(slab_ctx* ctx, double* time, double* dt, int32_t* frame, int64_t* steps);

/* Device-time breakdown since profiling was switched on, in milliseconds, per
 * kernel family: out[0] dt/control, [1] binning (tile descriptors), [2] P2G,
 * [3] grid update, [4] G2P (the next step's dt runs at its end).
 * Mirrors the reference's per-phase timers (src/simulation.cpp:512-519).
 * Enabled by slab_set_profiling(ctx, 1); adds event records per step. */
slab_status slab_set_profiling(slab_ctx* ctx, int32_t on);
slab_status slab_get_phase_times(slab_ctx* ctx, double out[5]);

/* Work done so far: out[0] = particle-steps (Np x completed steps),
 * out[1] = active node-steps (grid nodes with mass > 1e-6, summed over the
 * grid updates). These are the units of the roofline accounting. */
slab_status slab_work_counters(slab_ctx* ctx, int64_t out[2]);

/* FP32_SPLIT: CTA counts of the step's five work kernels now in use and the
 * tuning passes completed (as slab_batch_launch_shapes); zeros for FP64.
 * The shapes a context picks are remembered for the process, by device, tile
 * count and particle count (half-octave buckets): a later context of the same
 * size starts from them and measures none on its first steps (out[5] stays 0
 * until its next tuning pass). Shapes never change results. */
slab_status slab_launch_shapes(slab_ctx* ctx, int32_t out[6]);

/* FP32_SPLIT: persistent steps for this context (as
 * slab_batch_set_persistent); kept across later uploads. SLAB_E_ARG for
 * FP64_PLAIN parameters. */
slab_status slab_set_persistent(slab_ctx* ctx, int32_t on, int64_t limit_cycles);

/* Number of kernels this context has launched since creation. */
int64_t slab_kernel_launches(const slab_ctx* ctx);

/* The message of the context's last failed call. With ctx NULL: the message
 * of the calling thread's last failed slab_create, which leaves no context. */
const char* slab_last_error(const slab_ctx* ctx);
void slab_destroy(slab_ctx* ctx);

/* ---- batched ensembles ---------------------------------------------------
 * Many release scenarios of uneven size on one shared terrain, each with its
 * own slab_params (friction law and coefficients, total_time, dt_max, ...),
 * advanced together by the FP32 split step: every kernel launch covers all
 * running scenarios, each with its own adaptive dt (Simulation::updateDt per
 * scenario), replayed from CUDA graphs. A scenario's results are bitwise the
 * same as running it alone through slab_ctx with SLAB_FP32_SPLIT. There is
 * no reference counterpart: the reference runs one scenario per process
 * (src/main.cpp:29-57). */
typedef struct slab_batch slab_batch;

/* capacity_hint: node blocks (8x8 nodes, 2.8 KB each) to reserve up front,
 * 0 = automatic; the pool grows as scenarios spread. */
slab_status slab_batch_create(const slab_terrain_desc* terrain, const double* z, int32_t max_scenarios, int64_t capacity_hint,
                              slab_batch** out);
slab_status slab_batch_set_stream(slab_batch* b, void* cuda_stream);
/* Add a scenario (arrays as slab_upload_particles); params->precision must be
 * SLAB_FP32_SPLIT. Its t=0 pass runs with the next slab_batch_run. */
slab_status slab_batch_add(slab_batch* b, const slab_params* params, int32_t Np, const double* x_xy, const double* v_xy,
                           const double* vz, const double* h, const double* A, const double* mass, const double* z, int32_t* scenario_id);
/* Advance every scenario until each has reached its total_time, or for at
 * most max_steps steps of the batch. */
/* Add a scenario whose particles are built on the device from a release
 * (as slab_upload_release; the same particles as the reference's setup). */
slab_status slab_batch_add_release(slab_batch* b, const slab_params* params, const slab_release* release, int32_t* scenario_id);
slab_status slab_batch_run(slab_batch* b, int64_t max_steps, int64_t* steps_out);
slab_status slab_batch_state(slab_batch* b, int32_t scenario_id, double* time, int32_t* frame, int64_t* steps);
/* The scenario's own outcome: SLAB_OK, or the error that stopped it
 * (SLAB_E_DOMAIN, SLAB_E_NONFINITE, SLAB_E_OOM). A failed scenario stops at
 * once; the others run on, and slab_batch_run reports the first failure. */
slab_status slab_batch_scenario_status(slab_batch* b, int32_t scenario_id);
slab_status slab_batch_download_particles(slab_batch* b, int32_t scenario_id, double* x_xy, double* v_xy, double* vz, double* h,
                                          double* A, double* mass, double* z);
slab_status slab_batch_download_max(slab_batch* b, int32_t scenario_id, double* h_max, double* v_max2);
/* The scenario's particle moments, as slab_moments. */
slab_status slab_batch_moments(slab_batch* b, int32_t scenario_id, double out[6]);
/* The node box {i0, i1, j0, j1} a scenario's flow has touched and, when the
 * map pointers are not NULL and the box has at most cap_nodes nodes, h_max
 * and v_max2 over that box ((i-i0)*(j1-j0+1) + (j-j0)); an empty box has
 * i1 < i0. */
slab_status slab_batch_download_max_box(slab_batch* b, int32_t scenario_id, int32_t box[4], double* h_max, double* v_max2,
                                        int64_t cap_nodes);
/* The scenario's particle count (-1 for an unknown scenario). */
int32_t slab_batch_scenario_particles(const slab_batch* b, int32_t scenario_id);
/* out[0] = particle-steps, out[1] = active node-steps, over all scenarios. */
slab_status slab_batch_work_counters(slab_batch* b, int64_t out[2]);
int64_t slab_batch_kernel_launches(const slab_batch* b);
/* Per-kernel device times of the batch's steps, as slab_set_profiling /
 * slab_get_phase_times (adds event records per step while on). */
slab_status slab_batch_set_profiling(slab_batch* b, int32_t on);
slab_status slab_batch_phase_times(slab_batch* b, double out[5]);
/* Launch shapes (CTA counts) of the step's five work kernels: k_prep, P2G of
 * the dense tiles, P2G of the sparse tiles, grid update, G2P. Any shape gives
 * bitwise the same results. A tuner times five candidates per kernel (1/4,
 * 1/2, 1, 2 and 4 times the occupancy grid) on live, interleaved steps and keeps
 * the fastest; it runs on the first steps, after 4x as many steps as at its
 * last pick, and when the active tile count halves or doubles.
 * out[0..4] = the grids in use, out[5] = tuning passes completed. */
slab_status slab_batch_launch_shapes(slab_batch* b, int32_t out[6]);
/* grids[k] > 0 fixes kernel k's CTA count, 0 leaves it to the tuner (grids
 * NULL: none fixed); tune = 0 stops the tuner (shapes stay as they are). */
slab_status slab_batch_set_launch_shapes(slab_batch* b, const int32_t grids[5], int32_t tune);
/* Persistent steps (on = 1): each chunk of up to 32 steps becomes ONE
 * cooperative launch of a kernel that runs the step's phases (tile
 * bookkeeping, both P2G classes, grid update, G2P, end of step) for every
 * scenario, separated by grid-wide barriers instead of kernel boundaries, and
 * ends early once no scenario has work. The results are bitwise those of the
 * default path (separate kernels in CUDA graphs). Every barrier wait gives up
 * after limit_cycles SM clock cycles (0: keep the current limit, by default
 * 4e9, about two seconds): the waiting CTAs leave the kernel and every
 * scenario fails with SLAB_E_TIMEOUT, the device stays usable. The launch
 * shapes are then fixed (as many CTAs as fit on the device at once) and the
 * tuner does not run. SLAB_E_ARG if the device cannot launch cooperatively.
 * The environment variable SLAB_PERSIST=1 turns it on for every engine. */
slab_status slab_batch_set_persistent(slab_batch* b, int32_t on, int64_t limit_cycles);
const char* slab_batch_last_error(const slab_batch* b);
void slab_batch_destroy(slab_batch* b);

/* ---- serving -------------------------------------------------------------
 * A request loop with continuous batching. Submitted scenario solves wait in
 * a queue; a worker thread that owns the GPU admits them into free scenario
 * slots while their estimated HBM footprint fits the budget, runs them in
 * chunks of batched steps together with every other running scenario (each
 * with its own dt and friction), keeps their state on the device until they
 * reach total_time, then stores the result in host memory and frees the
 * slot. Results are bitwise the same as a solo FP32_SPLIT run. No reference
 * counterpart (the reference is a single-scenario CLI, src/main.cpp:29-57). */
typedef struct slab_server slab_server;
typedef struct slab_server_config {
    int32_t max_scenarios;    /* concurrent scenario slots */
    int32_t chunk_steps;      /* batched steps between admissions (0 = 32) */
    int64_t hbm_budget_bytes; /* admission budget (0 = half the free memory at creation) */
} slab_server_config;

/* request states reported by slab_server_poll */
enum { SLAB_REQ_QUEUED = 0, SLAB_REQ_RUNNING = 1, SLAB_REQ_DONE = 2, SLAB_REQ_CANCELLED = 3, SLAB_REQ_FAILED = 4 };

slab_status slab_server_create(const slab_terrain_desc* terrain, const double* z, const slab_server_config* config, slab_server** out);
/* Copy a scenario into the queue and return at once (params->precision must
 * be SLAB_FP32_SPLIT; arrays as slab_upload_particles). */
slab_status slab_server_submit(slab_server* s, const slab_params* params, int32_t Np, const double* x_xy, const double* v_xy,
                               const double* vz, const double* h, const double* A, const double* mass, const double* z, int64_t* request_id);
/* Queue a scenario given as a release: its particles are built on the
 * device when it is admitted (as slab_upload_release), so the setup is part
 * of the time to result and costs no host work. */
slab_status slab_server_submit_release(slab_server* s, const slab_params* params, const slab_release* release, int64_t* request_id);
/* The request's particle count (known for a release once it is admitted). */
slab_status slab_server_particles(slab_server* s, int64_t request_id, int32_t* Np);
slab_status slab_server_poll(slab_server* s, int64_t request_id, int32_t* state, double* seconds_to_result);
/* Block until the request is done (SLAB_E_TIMEOUT after timeout_s). */
slab_status slab_server_wait(slab_server* s, int64_t request_id, double timeout_s);
/* Result of a finished request: the node box {i0, i1, j0, j1} covered by its
 * flow, h_max and v_max2 over that box ((i-i0)*(j1-j0+1) + (j-j0); at most
 * cap_nodes), the final particles in upload order (any pointer may be NULL),
 * and info = {steps, simulated time, seconds to result, seconds queued}. */
slab_status slab_server_result(slab_server* s, int64_t request_id, int32_t box[4], double* h_max, double* v_max2, int64_t cap_nodes,
                               double* x_xy, double* v_xy, double* h, double* mass, double* info);
slab_status slab_server_cancel(slab_server* s, int64_t request_id);
/* Wait until no request is queued or running. */
slab_status slab_server_drain(slab_server* s, double timeout_s);
/* out = {completed, p50 and p99 seconds to result, completed per second
 * since the first submission, particle-steps, batched steps, seconds the
 * worker was busy, bytes admitted now}. */
slab_status slab_server_stats(slab_server* s, double out[8]);
/* Where the worker thread's time went: out = {seconds admitting requests
 * (host binning and uploads), seconds in chunks of batched steps (enqueue to
 * completion), seconds retiring finished requests (downloads, releases),
 * chunks run, mean and max scenarios running per chunk, capacity growths,
 * kernel launches}. */
slab_status slab_server_timing(slab_server* s, double out[8]);
const char* slab_server_last_error(const slab_server* s);
void slab_server_destroy(slab_server* s);

/* ---- setup utilities (host only; no device work) ---------------------- */

/* Poisson-disk samples in [0,Lx] x [0,Ly] with minimum distance r and k
 * candidates per active sample: the sampler of POISSON release sampling
 * (class Poisson_disk, src/poisson_disk_sampling.hpp:23-134). seed 0 draws
 * from the C library's rand() seeded with 1 -- the sequence the reference
 * consumes -- so it reproduces the reference's samples; any other seed uses a
 * seeded generator of this library. Positions are relative to the lower-left
 * corner, as the reference returns them. With out_xy == NULL only *n_out is
 * set; otherwise cap must be >= *n_out. */
slab_status slab_poisson_disk(double Lx, double Ly, double r, int32_t k, uint64_t seed, double* out_xy, int64_t cap, int64_t* n_out);

/* ---- frame-0 grid without allocation ----------------------------------- */

/* Largest node box slab_initial_grid_static accepts (e.g. 256 x 256). */
#define SLAB_STATIC_MAX_NODES 65536

/* No counterpart in the reference: an addition of this library for callers
 * that cannot allocate device memory -- a host framework that reserves the
 * whole GPU heap itself and forbids cudaMalloc/cudaFree by libraries, or a
 * real-time loop that may not allocate once running.
 *
 * Computes the grid of simulate()'s t=0 pass (P2G and the grid update with
 * dt = 0) with the FP32 split arithmetic, from particle arrays the caller
 * already has on the device, into device arrays the caller provides. It
 * makes no allocation: its scratch is a fixed array compiled into the
 * library (SLAB_STATIC_MAX_NODES nodes, about 3.9 MB per GPU). The array is
 * reserved on a device when the library's code is first loaded there: under
 * CUDA's default lazy module loading that is this entry point's first call
 * on the device (its first launch or symbol lookup), which can then fail
 * with SLAB_E_CUDA if the heap is already full. Make a first call (Np = 0
 * will do) before reserving the heap, or set CUDA_MODULE_LOADING=EAGER so
 * the array is reserved when the library loads. It stays reserved until
 * the process exits.
 *  - d_z: terrain heights on the device, Nx*Ny, i*Ny + j.
 *  - d_x_xy, d_v_xy (interleaved), d_vz, d_h, d_mass: Np particles.
 *  - box = {i0, i1, j0, j1}: the inclusive node box of the outputs; every
 *    particle's 3x3 stencil must lie inside it (else SLAB_E_DOMAIN), at
 *    most SLAB_STATIC_MAX_NODES nodes (larger boxes are rejected with
 *    SLAB_E_ARG).
 *  - outputs (device, box nodes, flattened (i-i0)*(j1-j0+1) + (j-j0)):
 *    normalised flow height, grid mass, velocity (interleaved), vz.
 *  - stream: a cudaStream_t or NULL. The call ends by waiting for the
 *    stream (it reads back an error flag), so it cannot be recorded into a
 *    CUDA graph by stream capture.
 * The first call on a device also looks up the device address of the
 * scratch array. All calls share the scratch and each clears the part it
 * uses first: calls that overlap on the GPU (other threads, other streams)
 * race and must be serialised by the caller. On error slab_last_error(NULL)
 * gives the message. */
slab_status slab_initial_grid_static(const slab_terrain_desc* terrain, const double* d_z, const slab_params* params, int32_t Np,
                                     const double* d_x_xy, const double* d_v_xy, const double* d_vz, const double* d_h, const double* d_mass,
                                     const int32_t box[4], double* d_h_out, double* d_mass_out, double* d_v_out, double* d_vz_out,
                                     void* stream);

/* Library version string and status-code names. */
const char* slab_version(void);
const char* slab_status_name(slab_status s);

#ifdef __cplusplus
}
#endif
#endif /* SLAB_GPU_H */
