/* CPU oracle: a plain-C restatement of the Slab-Pro depth-averaged MPM step
 * loop in FP64. TEST INFRASTRUCTURE ONLY -- the tests, the smoke check and the
 * CPU-baseline leg of bench.py call it as the checker; the product never
 * links it.
 *
 * Every function follows the reference operation for operation (same loop
 * order, same IEEE operations, no fused multiply-add), so that, built with
 * -ffp-contract=off, it reproduces the reference binary bit for bit. The
 * reference files cited are under src/ of ALMO-SLF-ETH/Slab-Pro.
 */
#ifndef SLAB_ORACLE_H
#define SLAB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_COULOMB = 0, ORACLE_VOELLMY = 1, ORACLE_MU_I = 2 };

typedef struct oracle_params {
    double gravity, rho;
    double C_cfl, dt_max, flip_ratio;
    double output_dt, total_time;
    int32_t friction_type; /* ORACLE_* */
    int32_t sort_period;   /* 50 in the reference (simulation.cpp:540); 0 = never */
    double coulomb_mu;
    double voellmy_mu, voellmy_xi;
    double mui_mu1, mui_mu2, mui_I0, mui_d, mui_phi;
} oracle_params;

typedef struct oracle_sim oracle_sim;

/* Terrain z is given as z[i*Ny + j] (tools.hpp:172 ind()), node x = i*dx,
 * y = j*dx. Computes the cell gradients and slope angles
 * (complex_terrain.cpp:84-111) and zeroes h_max / v_max2. */
oracle_sim* oracle_create(const oracle_params* p, int32_t Nx, int32_t Ny, double dx, const double* z);
void oracle_destroy(oracle_sim* s);

/* Particle arrays as in data_arrays.hpp: x and v interleaved (x0,y0,x1,...). */
int oracle_set_particles(oracle_sim* s, int32_t Np, const double* x, const double* z, const double* v, const double* vz, const double* h,
                         const double* A, const double* mass, const double* theta);

/* simulate()'s t=0 pass: remesh, P2G, computeGridVelocity with dt = 0
 * (simulation.cpp:493-495). Returns 0 or a negative error. */
int oracle_t0(oracle_sim* s);

/* One iteration of simulate()'s while loop (simulation.cpp:500-510):
 * advanceStep, time += dt, frame bump. Returns 1 if a frame was completed,
 * 0 if not, negative on error (-1: particle stencil left the terrain). */
int oracle_step(oracle_sim* s);

/* Run oracle_step until time >= total_time or max_steps steps. Returns the
 * number of steps taken or a negative error. */
int64_t oracle_run(oracle_sim* s, int64_t max_steps);

void oracle_get_state(const oracle_sim* s, double* time, double* dt, int32_t* frame, int64_t* step);
void oracle_get_particles(const oracle_sim* s, double* x, double* z, double* v, double* vz, double* h, double* A, double* mass, double* theta);
/* grid header: Nx, Ny, i_off, j_off (the remeshed bounding box) */
void oracle_get_grid_dims(const oracle_sim* s, int32_t* dims4);
void oracle_get_grid(const oracle_sim* s, double* h, double* mass, double* v, double* vz, double* flip);
/* Grid::F (P2G force sums) and Grid::a = F / mass over the same box,
 * interleaved (x, y) */
void oracle_get_grid_force(const oracle_sim* s, double* F, double* a);
void oracle_get_max(const oracle_sim* s, double* h_max, double* v_max2);
/* upload index of each particle in the current (block-sorted) order */
void oracle_get_ids(const oracle_sim* s, int32_t* ids);
void oracle_get_terrain_metrics(const oracle_sim* s, double* grad, double* theta);

#ifdef __cplusplus
}
#endif
#endif
