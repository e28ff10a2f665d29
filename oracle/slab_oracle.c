/* CPU oracle: plain-C restatement of the Slab-Pro FP64 step loop.
 * TEST INFRASTRUCTURE ONLY (see slab_oracle.h). Parity pinned: the tests
 * compare it bit for bit with the reference's own sources built unmodified
 * into oracle/_ref/slab_ref and with the golden fixtures in tests/golden/.
 *
 * Citations are to src/ of ALMO-SLF-ETH/Slab-Pro. Expressions are written
 * with the same association as the reference (C evaluates a*b*c as (a*b)*c
 * like C++), and 2-vector operations component by component, as Eigen does.
 */
#include "slab_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct oracle_sim {
    oracle_params p;
    int Nx, Ny;
    double dx, one_over_dx;
    /* terrain (data_arrays.hpp:49-93, full DEM) */
    double *tx, *ty, *tz, *tgx, *tgy, *ttheta, *h_max, *v_max2;
    /* particles (data_arrays.hpp:22-47) */
    int Np;
    double *px, *py, *pz, *pvx, *pvy, *pvz, *ph, *pA, *pm, *pth;
    int* order;
    int* pid; /* upload index of each particle, permuted with it (not in the reference) */
    /* remeshed grid (simulation.cpp:584-642) */
    int gNx, gNy, gi0, gj0;
    size_t gcap;
    double *gz, *gh, *gm, *gFx, *gFy, *gflx, *gfly, *gvx, *gvy, *gvz;
    /* time stepping (simulation.hpp:303-310) */
    double time, dt;
    int frame;
    int64_t step;
};

static inline int ind(int i, int j, int Ny) { return i * Ny + j; } /* tools.hpp:172-174 */

static inline int sgn(double v) { return (0.0 < v) - (v < 0.0); } /* tools.hpp:90-92 */

/* quadratic B-spline, tools.hpp:119-128 */
static inline double N(double u) {
    double uabs = fabs(u);
    if (uabs < 0.5) return 0.75 - uabs * uabs;
    if (uabs < 1.5) return 0.5 * (1.5 - uabs) * (1.5 - uabs);
    return 0.0;
}

/* its derivative, tools.hpp:131-140 */
static inline double dNdu(double u) {
    double uabs = fabs(u);
    if (uabs < 0.5) return (-2.0 * u);
    if (uabs < 1.5) return (u - 1.5 * (double)sgn(u));
    return 0.0;
}

static double* dalloc(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }

oracle_sim* oracle_create(const oracle_params* p, int32_t Nx, int32_t Ny, double dx, const double* z) {
    oracle_sim* s = (oracle_sim*)calloc(1, sizeof(oracle_sim));
    if (!s) return NULL;
    s->p = *p;
    s->Nx = Nx;
    s->Ny = Ny;
    s->dx = dx;
    s->one_over_dx = 1. / dx;
    size_t n = (size_t)Nx * Ny;
    s->tx = dalloc(Nx);
    s->ty = dalloc(Ny);
    for (int i = 0; i < Nx; ++i) s->tx[i] = (double)i * dx; /* complex_terrain.cpp:49-53, 67-82 */
    for (int j = 0; j < Ny; ++j) s->ty[j] = (double)j * dx;
    s->tz = dalloc(n);
    memcpy(s->tz, z, n * sizeof(double));
    s->tgx = dalloc(n);
    s->tgy = dalloc(n);
    s->ttheta = dalloc(n);
    s->h_max = dalloc(n);
    s->v_max2 = dalloc(n);
    /* terrainGradients, complex_terrain.cpp:84-100: cell gradient stored at
     * the bottom-left node; last row and column stay zero */
    const double ood = s->one_over_dx;
    for (int i = 0; i < Nx - 1; ++i) {
        for (int j = 0; j < Ny - 1; ++j) {
            const double* t = s->tz;
            double dz_x = (t[ind(i + 1, j, Ny)] + t[ind(i + 1, j + 1, Ny)] - t[ind(i, j, Ny)] - t[ind(i, j + 1, Ny)]) / 2. * ood;
            double dz_y = (t[ind(i, j + 1, Ny)] + t[ind(i + 1, j + 1, Ny)] - t[ind(i, j, Ny)] - t[ind(i + 1, j, Ny)]) / 2. * ood;
            s->tgx[ind(i, j, Ny)] = dz_x;
            s->tgy[ind(i, j, Ny)] = dz_y;
        }
    }
    /* terrainTheta, complex_terrain.cpp:102-111 */
    for (size_t k = 0; k < n; ++k) s->ttheta[k] = atan(sqrt(s->tgx[k] * s->tgx[k] + s->tgy[k] * s->tgy[k]));
    return s;
}

void oracle_destroy(oracle_sim* s) {
    if (!s) return;
    double* arrs[] = {s->tx, s->ty, s->tz, s->tgx, s->tgy, s->ttheta, s->h_max, s->v_max2, s->px, s->py, s->pz, s->pvx, s->pvy,
                      s->pvz, s->ph, s->pA, s->pm, s->pth, s->gz, s->gh, s->gm, s->gFx, s->gFy, s->gflx, s->gfly, s->gvx, s->gvy, s->gvz};
    for (size_t k = 0; k < sizeof arrs / sizeof arrs[0]; ++k) free(arrs[k]);
    free(s->order);
    free(s->pid);
    free(s);
}

int oracle_set_particles(oracle_sim* s, int32_t Np, const double* x, const double* z, const double* v, const double* vz, const double* h,
                         const double* A, const double* mass, const double* theta) {
    if (Np <= 0) return -2;
    s->Np = Np;
    double** a[] = {&s->px, &s->py, &s->pz, &s->pvx, &s->pvy, &s->pvz, &s->ph, &s->pA, &s->pm, &s->pth};
    for (size_t k = 0; k < sizeof a / sizeof a[0]; ++k) {
        free(*a[k]);
        *a[k] = dalloc(Np);
    }
    free(s->order);
    s->order = (int*)calloc(Np, sizeof(int));
    free(s->pid);
    s->pid = (int*)calloc(Np, sizeof(int));
    for (int p = 0; p < Np; ++p) {
        s->px[p] = x[2 * p];
        s->py[p] = x[2 * p + 1];
        s->pvx[p] = v[2 * p];
        s->pvy[p] = v[2 * p + 1];
        s->pz[p] = z[p];
        s->pvz[p] = vz[p];
        s->ph[p] = h[p];
        s->pA[p] = A[p];
        s->pm[p] = mass[p];
        s->pth[p] = theta[p];
        s->order[p] = p;
        s->pid[p] = p;
    }
    s->time = 0.0;
    s->dt = 0.0; /* simulation.hpp:39: dt starts at zero for the t=0 pass */
    s->frame = 0;
    s->step = 0;
    return 0;
}

/* particleGradients / particleSlopeAngle, complex_terrain.cpp:113-130:
 * values of the cell that contains the particle (floor index) */
static inline int cell_of(const oracle_sim* s, int p) {
    int i_base = (int)floor((s->px[p] - s->tx[0]) * s->one_over_dx);
    int j_base = (int)floor((s->py[p] - s->ty[0]) * s->one_over_dx);
    return ind(i_base, j_base, s->Ny);
}

/* updateDt, simulation.cpp:565-582 */
static void update_dt(oracle_sim* s) {
    int imax = 0;
    double best = s->pvx[0] * s->pvx[0] + s->pvy[0] * s->pvy[0];
    for (int p = 1; p < s->Np; ++p) { /* std::max_element: first of equal maxima */
        double sq = s->pvx[p] * s->pvx[p] + s->pvy[p] * s->pvy[p];
        if (best < sq) {
            best = sq;
            imax = p;
        }
    }
    double max_speed = sqrt(s->pvx[imax] * s->pvx[imax] + s->pvy[imax] * s->pvy[imax]);
    if (max_speed > 0.0) {
        double a = s->p.C_cfl * s->dx / max_speed;
        s->dt = (s->p.dt_max < a) ? s->p.dt_max : a; /* std::min */
    } else {
        s->dt = s->p.dt_max;
    }
    double next_frame_time = s->p.output_dt * (s->frame + 1);
    if (s->time + s->dt > next_frame_time - 1e-12) s->dt = next_frame_time - s->time;
}

/* remesh, simulation.cpp:584-642 */
static int remesh(oracle_sim* s) {
    double min_x = s->px[0], max_x = s->px[0], min_y = s->py[0], max_y = s->py[0];
    for (int p = 1; p < s->Np; ++p) {
        if (s->px[p] < min_x) min_x = s->px[p];
        if (!(s->px[p] < max_x)) max_x = s->px[p];
        if (s->py[p] < min_y) min_y = s->py[p];
        if (!(s->py[p] < max_y)) max_y = s->py[p];
    }
    const double epsilon = 1e-8 * s->dx;
    int il = (int)((min_x - s->tx[0]) * s->one_over_dx - 1.0 - epsilon);
    int ir = (int)((max_x - s->tx[0]) * s->one_over_dx + 2.0 + epsilon);
    int jb = (int)((min_y - s->ty[0]) * s->one_over_dx - 1.0 - epsilon);
    int jt = (int)((max_y - s->ty[0]) * s->one_over_dx + 2.0 + epsilon);
    /* the reference does not check this; indexing past the terrain is
     * undefined behaviour there */
    if (il < 0 || jb < 0 || ir > s->Nx - 1 || jt > s->Ny - 1) return -1;
    s->gi0 = il;
    s->gj0 = jb;
    s->gNx = ir - il + 1;
    s->gNy = jt - jb + 1;
    size_t n = (size_t)s->gNx * s->gNy;
    if (n > s->gcap) {
        double** a[] = {&s->gz, &s->gh, &s->gm, &s->gFx, &s->gFy, &s->gflx, &s->gfly, &s->gvx, &s->gvy, &s->gvz};
        for (size_t k = 0; k < sizeof a / sizeof a[0]; ++k) {
            free(*a[k]);
            *a[k] = dalloc(n);
        }
        s->gcap = n;
    }
    memset(s->gh, 0, n * sizeof(double));
    memset(s->gm, 0, n * sizeof(double));
    memset(s->gFx, 0, n * sizeof(double));
    memset(s->gFy, 0, n * sizeof(double));
    memset(s->gflx, 0, n * sizeof(double));
    memset(s->gfly, 0, n * sizeof(double));
    memset(s->gvx, 0, n * sizeof(double));
    memset(s->gvy, 0, n * sizeof(double));
    memset(s->gvz, 0, n * sizeof(double));
    for (int i = il; i <= ir; ++i)
        for (int j = jb; j <= jt; ++j) s->gz[ind(i - il, j - jb, s->gNy)] = s->tz[ind(i, j, s->Ny)];
    return 0;
}

/* sort_particles_by_grid_block + apply_particle_permutation,
 * simulation.cpp:644-724: stable counting sort by 4x4 node block */
static void sort_by_block(oracle_sim* s) {
    const int B = 4;
    const int nbx = (s->gNx + B - 1) / B, nby = (s->gNy + B - 1) / B, nblocks = nbx * nby;
    const double gx0 = s->tx[s->gi0], gy0 = s->ty[s->gj0];
    int* counts = (int*)calloc(nblocks, sizeof(int));
    int* bid = (int*)calloc(s->Np, sizeof(int));
    for (int p = 0; p < s->Np; ++p) {
        int ib = (int)((s->px[p] - gx0) * s->one_over_dx - 0.5);
        int jb = (int)((s->py[p] - gy0) * s->one_over_dx - 0.5);
        if (ib < 0) ib = 0;
        if (jb < 0) jb = 0;
        if (ib >= s->gNx) ib = s->gNx - 1;
        if (jb >= s->gNy) jb = s->gNy - 1;
        int b = (ib / B) * nby + jb / B;
        bid[p] = b;
        counts[b]++;
    }
    int* next = (int*)calloc(nblocks, sizeof(int));
    int sum = 0;
    for (int b = 0; b < nblocks; ++b) {
        next[b] = sum;
        sum += counts[b];
    }
    for (int p = 0; p < s->Np; ++p) s->order[next[bid[p]]++] = p;
    double* tmp = dalloc(s->Np);
    double* arrs[] = {s->px, s->py, s->pz, s->pvx, s->pvy, s->pvz, s->ph, s->pA, s->pm, s->pth};
    for (size_t k = 0; k < sizeof arrs / sizeof arrs[0]; ++k) {
        for (int q = 0; q < s->Np; ++q) tmp[q] = arrs[k][s->order[q]];
        memcpy(arrs[k], tmp, s->Np * sizeof(double));
    }
    int* itmp = (int*)calloc(s->Np, sizeof(int));
    for (int q = 0; q < s->Np; ++q) itmp[q] = s->pid[s->order[q]];
    memcpy(s->pid, itmp, s->Np * sizeof(int));
    free(itmp);
    free(tmp);
    free(next);
    free(bid);
    free(counts);
}

/* P2G, simulation.cpp:726-798 */
static void p2g(oracle_sim* s) {
    const double ood = s->one_over_dx, g = s->p.gravity, rho = s->p.rho;
    const int gNy = s->gNy;
    const double gx0 = s->tx[s->gi0], gy0 = s->ty[s->gj0];
    for (int p = 0; p < s->Np; ++p) {
        const double xp = s->px[p], yp = s->py[p];
        const double height_p = s->ph[p], A_p = s->pA[p];
        const double vx = s->pvx[p], vy = s->pvy[p];
        const double m_p = s->pm[p];
        const double vmx = vx * m_p, vmy = vy * m_p;
        const double vzm_p = s->pvz[p] * m_p;
        const double hm_p = height_p * m_p;
        const double h_A = height_p * A_p;
        const int i_base = (int)((xp - gx0) * ood - 0.5);
        const int j_base = (int)((yp - gy0) * ood - 0.5);
        const int c = cell_of(s, p);
        const double gradx = s->tgx[c], grady = s->tgy[c];
        s->pth[p] = s->ttheta[c];
        const double cos_t = cos(s->pth[p]);
        const double coeff = -m_p * g * cos_t * cos_t;
        const double m_b_px = coeff * gradx, m_b_py = coeff * grady;
        const double s00 = -0.5 * rho * g * cos_t * cos_t * height_p, s11 = s00, s01 = 0.0, s10 = 0.0;
        double wx[3], wy[3], dwx[3], dwy[3];
        for (int d = 0; d < 3; ++d) {
            double ux = (xp - s->tx[s->gi0 + i_base + d]) * ood;
            wx[d] = N(ux);
            dwx[d] = dNdu(ux) * ood;
            double uy = (yp - s->ty[s->gj0 + j_base + d]) * ood;
            wy[d] = N(uy);
            dwy[d] = dNdu(uy) * ood;
        }
        for (int di = 0; di < 3; ++di) {
            for (int dj = 0; dj < 3; ++dj) {
                const double weight = wx[di] * wy[dj];
                if (weight > 3e-3) {
                    const double gwx = dwx[di] * wy[dj];
                    const double gwy = dwy[dj] * wx[di];
                    const int k = ind(i_base + di, j_base + dj, gNy);
                    s->gm[k] += m_p * weight;
                    s->gvx[k] += vmx * weight;
                    s->gvy[k] += vmy * weight;
                    s->gvz[k] += vzm_p * weight;
                    s->gh[k] += hm_p * weight;
                    s->gFx[k] += m_b_px * weight - h_A * (s00 * gwx + s01 * gwy);
                    s->gFy[k] += m_b_py * weight - h_A * (s11 * gwy + s10 * gwx);
                }
            }
        }
    }
}

/* computeGridVelocity, simulation.cpp:800-875 */
static void grid_velocity(oracle_sim* s) {
    const double g = s->p.gravity, dt = s->dt;
    for (int i = 0; i < s->gNx; ++i) {
        for (int j = 0; j < s->gNy; ++j) {
            const int k = ind(i, j, s->gNy);
            const double m_i = s->gm[k];
            if (m_i > 1e-6) {
                s->gvx[k] /= m_i;
                s->gvy[k] /= m_i;
                s->gvz[k] /= m_i;
                s->gh[k] /= m_i;
                const double vox = s->gvx[k], voy = s->gvy[k];
                const double ax = s->gFx[k] / m_i, ay = s->gFy[k] / m_i;
                const double vtx = vox + dt * ax, vty = voy + dt * ay;
                const double v_sq = vtx * vtx + vty * vty;
                const int t = ind(s->gi0 + i, s->gj0 + j, s->Ny);
                if (v_sq > 1e-16) {
                    const double gx = s->tgx[t], gy = s->tgy[t];
                    const double cos_theta = cos(s->ttheta[t]);
                    const double v_z = vtx * gx + vty * gy;
                    const double v_3D_sq = v_sq + v_z * v_z;
                    const double v_norm_3D = sqrt(v_3D_sq);
                    double a_fric = 0.;
                    const double hk = s->gh[k];
                    switch (s->p.friction_type) {
                        case ORACLE_COULOMB:
                            a_fric = s->p.coulomb_mu * g * cos_theta;
                            break;
                        case ORACLE_VOELLMY:
                            a_fric = s->p.voellmy_mu * g * cos_theta + g * v_3D_sq / (s->p.voellmy_xi * hk * cos_theta);
                            break;
                        case ORACLE_MU_I: {
                            const double I = 5. * s->p.mui_d * v_norm_3D / (2. * hk * cos_theta * cos_theta * sqrt(g * hk * s->p.mui_phi));
                            const double mu_I = s->p.mui_mu1 + (s->p.mui_mu2 - s->p.mui_mu1) / (1. + s->p.mui_I0 / I);
                            a_fric = mu_I * g * cos_theta;
                            break;
                        }
                    }
                    const double dv = dt * a_fric;
                    if (dv < v_norm_3D) {
                        const double f = 1. - dv / v_norm_3D;
                        s->gvx[k] = vtx * f;
                        s->gvy[k] = vty * f;
                    } else {
                        s->gvx[k] = 0.0;
                        s->gvy[k] = 0.0;
                    }
                } else {
                    s->gvx[k] = 0.0;
                    s->gvy[k] = 0.0;
                }
                s->gflx[k] = s->gvx[k] - vox;
                s->gfly[k] = s->gvy[k] - voy;
                if (s->h_max[t] < s->gh[k]) s->h_max[t] = s->gh[k]; /* std::max */
                const double v2 = s->gvx[k] * s->gvx[k] + s->gvy[k] * s->gvy[k];
                if (s->v_max2[t] < v2) s->v_max2[t] = v2;
            } else {
                s->gvx[k] = 0.0;
                s->gvy[k] = 0.0;
                s->gvz[k] = 0.;
                s->gh[k] = 0.;
            }
        }
    }
}

/* G2P, simulation.cpp:877-940 */
static void g2p(oracle_sim* s) {
    const double ood = s->one_over_dx, dt = s->dt, fr = s->p.flip_ratio, rho = s->p.rho;
    const int gNy = s->gNy;
    const double gx0 = s->tx[s->gi0], gy0 = s->ty[s->gj0];
    for (int p = 0; p < s->Np; ++p) {
        const int c = cell_of(s, p);
        const double pgx = s->tgx[c], pgy = s->tgy[c];
        const double xp = s->px[p], yp = s->py[p];
        const int i_base = (int)((xp - gx0) * ood - 0.5);
        const int j_base = (int)((yp - gy0) * ood - 0.5);
        double picx = 0.0, picy = 0.0, flx = 0.0, fly = 0.0, z_p = 0.;
        double wx[3], wy[3], dwx[3], dwy[3];
        for (int d = 0; d < 3; ++d) {
            double ux = (xp - s->tx[s->gi0 + i_base + d]) * ood;
            wx[d] = N(ux);
            dwx[d] = dNdu(ux) * ood;
            double uy = (yp - s->ty[s->gj0 + j_base + d]) * ood;
            wy[d] = N(uy);
            dwy[d] = dNdu(uy) * ood;
        }
        double strain_trace = 0.;
        for (int di = 0; di < 3; ++di) {
            for (int dj = 0; dj < 3; ++dj) {
                const double weight = wx[di] * wy[dj];
                const int k = ind(i_base + di, j_base + dj, gNy);
                const double gwx = dwx[di] * wy[dj];
                const double gwy = dwy[dj] * wx[di];
                picx += s->gvx[k] * weight;
                picy += s->gvy[k] * weight;
                flx += s->gflx[k] * weight;
                fly += s->gfly[k] * weight;
                z_p += s->gz[k] * weight;
                strain_trace += gwx * s->gvx[k] + gwy * s->gvy[k];
            }
        }
        strain_trace *= dt;
        s->pz[p] = z_p;
        const double nvx = fr * (s->pvx[p] + flx) + (1. - fr) * picx;
        const double nvy = fr * (s->pvy[p] + fly) + (1. - fr) * picy;
        s->pvx[p] = nvx;
        s->pvy[p] = nvy;
        s->pvz[p] = nvx * pgx + nvy * pgy;
        s->px[p] = xp + dt * picx;
        s->py[p] = yp + dt * picy;
        s->ph[p] /= 1. + strain_trace;
        s->pA[p] = s->pm[p] / (s->ph[p] * rho);
    }
}

int oracle_t0(oracle_sim* s) {
    if (remesh(s)) return -1;
    p2g(s);
    grid_velocity(s);
    return 0;
}

int oracle_step(oracle_sim* s) {
    s->step++;
    /* advanceStep, simulation.cpp:524-563 */
    update_dt(s);
    if (remesh(s)) return -1;
    if (s->p.sort_period > 0 && s->step % s->p.sort_period == 0) sort_by_block(s);
    p2g(s);
    grid_velocity(s);
    g2p(s);
    s->time += s->dt;
    if (s->p.output_dt * (s->frame + 1) - s->time < 1e-13) {
        s->frame++;
        return 1;
    }
    return 0;
}

int64_t oracle_run(oracle_sim* s, int64_t max_steps) {
    int64_t n = 0;
    while (s->time < s->p.total_time && n < max_steps) {
        int r = oracle_step(s);
        if (r < 0) return r;
        ++n;
    }
    return n;
}

void oracle_get_state(const oracle_sim* s, double* time, double* dt, int32_t* frame, int64_t* step) {
    if (time) *time = s->time;
    if (dt) *dt = s->dt;
    if (frame) *frame = s->frame;
    if (step) *step = s->step;
}

void oracle_get_particles(const oracle_sim* s, double* x, double* z, double* v, double* vz, double* h, double* A, double* mass, double* theta) {
    for (int p = 0; p < s->Np; ++p) {
        if (x) {
            x[2 * p] = s->px[p];
            x[2 * p + 1] = s->py[p];
        }
        if (v) {
            v[2 * p] = s->pvx[p];
            v[2 * p + 1] = s->pvy[p];
        }
        if (z) z[p] = s->pz[p];
        if (vz) vz[p] = s->pvz[p];
        if (h) h[p] = s->ph[p];
        if (A) A[p] = s->pA[p];
        if (mass) mass[p] = s->pm[p];
        if (theta) theta[p] = s->pth[p];
    }
}

void oracle_get_grid_dims(const oracle_sim* s, int32_t* d) {
    d[0] = s->gNx;
    d[1] = s->gNy;
    d[2] = s->gi0;
    d[3] = s->gj0;
}

/* Grid::F as P2G leaves it (simulation.cpp:792-793) and Grid::a = F / m_i
 * where m_i > 1e-6 (simulation.cpp:807-814), zero elsewhere as remesh fills
 * it (simulation.cpp:626-627). */
void oracle_get_grid_force(const oracle_sim* s, double* F, double* a) {
    size_t n = (size_t)s->gNx * s->gNy;
    for (size_t k = 0; k < n; ++k) {
        const double m_i = s->gm[k];
        if (F) {
            F[2 * k] = s->gFx[k];
            F[2 * k + 1] = s->gFy[k];
        }
        if (a) {
            a[2 * k] = m_i > 1e-6 ? s->gFx[k] / m_i : 0.0;
            a[2 * k + 1] = m_i > 1e-6 ? s->gFy[k] / m_i : 0.0;
        }
    }
}

void oracle_get_grid(const oracle_sim* s, double* h, double* mass, double* v, double* vz, double* flip) {
    size_t n = (size_t)s->gNx * s->gNy;
    for (size_t k = 0; k < n; ++k) {
        if (h) h[k] = s->gh[k];
        if (mass) mass[k] = s->gm[k];
        if (vz) vz[k] = s->gvz[k];
        if (v) {
            v[2 * k] = s->gvx[k];
            v[2 * k + 1] = s->gvy[k];
        }
        if (flip) {
            flip[2 * k] = s->gflx[k];
            flip[2 * k + 1] = s->gfly[k];
        }
    }
}

void oracle_get_max(const oracle_sim* s, double* h_max, double* v_max2) {
    size_t n = (size_t)s->Nx * s->Ny;
    if (h_max) memcpy(h_max, s->h_max, n * sizeof(double));
    if (v_max2) memcpy(v_max2, s->v_max2, n * sizeof(double));
}

void oracle_get_terrain_metrics(const oracle_sim* s, double* grad, double* theta) {
    size_t n = (size_t)s->Nx * s->Ny;
    for (size_t k = 0; k < n; ++k) {
        if (grad) {
            grad[2 * k] = s->tgx[k];
            grad[2 * k + 1] = s->tgy[k];
        }
        if (theta) theta[k] = s->ttheta[k];
    }
}

void oracle_get_ids(const oracle_sim* s, int32_t* ids) {
    for (int p = 0; p < s->Np; ++p) ids[p] = s->pid[p];
}
