// Batched ensembles: many release scenarios of uneven size on one shared
// terrain, each with its own parameters, adaptive dt and friction law,
// advanced together by the FP32 split step (one launch per kernel per step
// for all scenarios, replayed from CUDA graphs). Results are bitwise the
// same as running each scenario alone through slab_ctx (FP32_SPLIT): a
// scenario's sums never mix with another's, and every sum has a fixed order
// or is exact.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "engine.hpp"
#include "engine32.hpp"
#include "release.hpp"

namespace slab {
void set_thread_error(const std::string& msg);
}

using namespace slab;

struct slab_batch {
    Terrain terrain;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    int max_scn = 0;
    Ctl* d_ctl = nullptr;  // [max_scn]
    Ctl* h_ctl = nullptr;  // pinned mirror
    std::unique_ptr<Engine32> E;
    std::vector<slab_params> params;
    std::vector<int> Np;
    int t0_done = 0;  // scenarios that have had their t=0 pass
    std::string err;
    int chunk = 32;
};

namespace {

template <typename F> slab_status bguard(slab_batch* b, F&& f) {
    try {
        f();
        if (b) b->err.clear();
        return SLAB_OK;
    } catch (const Error& e) {
        if (b) b->err = e.msg;
        set_thread_error(e.msg);
        return e.code;
    } catch (const std::exception& e) {
        if (b) b->err = e.what();
        set_thread_error(e.what());
        return SLAB_E_ARG;
    }
}

void bneed(bool ok, slab_status code, const char* msg) {
    if (!ok) throw Error{code, msg};
}

void pull_all(slab_batch* b) {
    const int n = b->E ? b->E->nscn : 0;
    if (n) SLAB_CUDA(cudaMemcpyAsync(b->h_ctl, b->d_ctl, n * sizeof(Ctl), cudaMemcpyDeviceToHost, b->stream));
    SLAB_CUDA(cudaStreamSynchronize(b->stream));
}

slab_status status_of(int e) {
    if (e & ERR_NONFINITE) return SLAB_E_NONFINITE;
    if (e & (ERR_DOMAIN | ERR_MOVE)) return SLAB_E_DOMAIN;
    if (e & ERR_CAPACITY) return SLAB_E_OOM;
    if (e & ERR_TIMEOUT) return SLAB_E_TIMEOUT;
    return SLAB_OK;
}

void raise_errors(slab_batch* b) {
    int nfail = 0, first = -1;
    for (int s = 0; s < b->E->nscn; ++s)
        if (status_of(b->h_ctl[s].err) != SLAB_OK) {
            if (first < 0) first = s;
            ++nfail;
        }
    if (first < 0) return;
    const slab_status code = status_of(b->h_ctl[first].err);
    const char* what = code == SLAB_E_NONFINITE ? "non-finite particle state"
                       : code == SLAB_E_DOMAIN  ? "a particle stencil left the terrain"
                                                : "device capacity exceeded";
    throw Error{code, "scenario " + std::to_string(first) + ": " + what + " (" + std::to_string(nfail) + " scenario(s) failed)"};
}

void run_t0(slab_batch* b) {
    if (b->t0_done < b->E->nscn) {
        b->E->launch_t0();
        b->t0_done = b->E->nscn;
    }
}

}  // namespace

extern "C" {

slab_status slab_batch_create(const slab_terrain_desc* td, const double* z, int32_t max_scenarios, int64_t capacity_hint,
                              slab_batch** out) {
    if (!td || !z || !out || max_scenarios <= 0) return SLAB_E_ARG;
    *out = nullptr;
    slab_batch* b = new slab_batch();
    slab_status s = bguard(b, [&] {
        bneed(td->Nx >= 4 && td->Ny >= 4 && std::isfinite(td->dx) && td->dx > 0, SLAB_E_ARG, "invalid terrain");
        bneed((int64_t)td->Nx * td->Ny < (int64_t(1) << 31), SLAB_E_ARG, "terrain too large");
        SLAB_CUDA(cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking));
        b->stream = b->own_stream;
        b->max_scn = max_scenarios;
        b->d_ctl = dmalloc<Ctl>(max_scenarios);
        SLAB_CUDA(cudaMallocHost(&b->h_ctl, max_scenarios * sizeof(Ctl)));
        Terrain& t = b->terrain;
        t.Nx = td->Nx;
        t.Ny = td->Ny;
        t.dx = td->dx;
        t.xll = td->xllcorner;
        t.yll = td->yllcorner;
        const size_t n = (size_t)t.Nx * t.Ny;
        t.z = dalloc<double>(n);
        t.grad = dalloc<double2>(n);
        t.cos_t = dalloc<double>(n);
        t.dem32 = dalloc<float4>(n);
        SLAB_CUDA(cudaMemcpyAsync(t.z.get(), z, n * sizeof(double), cudaMemcpyHostToDevice, b->stream));
        compute_terrain_metrics(t, b->stream);
        const int64_t ntiles = (int64_t)((t.Nx + TILE - 1) / TILE) * ((t.Ny + TILE - 1) / TILE);
        // node blocks are shared by all scenarios: default pool = the terrain's tiles times a few scenarios
        const int64_t blk = capacity_hint > 0 ? capacity_hint : std::min<int64_t>(ntiles, 1 << 16);
        b->E.reset(new Engine32(t, b->stream, max_scenarios, blk, true));
        SLAB_CUDA(cudaStreamSynchronize(b->stream));
    });
    if (s != SLAB_OK) {
        slab_batch_destroy(b);
        return s;
    }
    *out = b;
    return SLAB_OK;
}

namespace {
// a new scenario from host or device particle arrays
int batch_add_arrays(slab_batch* b, const slab_params* p, int32_t Np, const double* x, const double* v, const double* vz, const double* h,
                     const double* m, const double* z) {
    bneed(p->precision == SLAB_FP32_SPLIT, SLAB_E_ARG, "batches run the FP32_SPLIT arithmetic");
    bneed(b->E->nscn < b->max_scn, SLAB_E_OOM, "batch is full");
    const int sid = b->E->nscn;
    Ctl& c = b->h_ctl[sid];
    std::memset(&c, 0, sizeof(Ctl));
    c.dx = b->terrain.dx;
    c.one_over_dx = 1. / b->terrain.dx;
    c.C_cfl = p->C_cfl;
    c.dt_max = p->dt_max;
    c.output_dt = p->output_dt;
    c.total_time = p->total_time;
    c.stop = 1;
    const int got = b->E->add_scenario(*p, b->d_ctl + sid, &c, Np, x, v, vz, h, m, z);
    bneed(got == sid, SLAB_E_STATE, "scenario id mismatch");
    b->params.push_back(*p);
    b->Np.push_back(Np);
    return sid;
}
}  // namespace

slab_status slab_batch_add(slab_batch* b, const slab_params* p, int32_t Np, const double* x, const double* v, const double* vz,
                           const double* h, const double* A, const double* m, const double* z, int32_t* sid_out) {
    if (!b || !p) return SLAB_E_ARG;
    (void)A;
    return bguard(b, [&] {
        bneed(Np > 0 && x && v && vz && h && m && z, SLAB_E_ARG, "invalid particle arrays");
        for (int q = 0; q < Np; ++q) bneed(h[q] > 0 && m[q] > 0, SLAB_E_ARG, "particle h and mass must be > 0");
        const int sid = batch_add_arrays(b, p, Np, x, v, vz, h, m, z);
        if (sid_out) *sid_out = sid;
    });
}

slab_status slab_batch_add_release(slab_batch* b, const slab_params* p, const slab_release* r, int32_t* sid_out) {
    if (!b || !p || !r) return SLAB_E_ARG;
    return bguard(b, [&] {
        bneed(std::isfinite(p->rho) && p->rho > 0, SLAB_E_ARG, "rho must be > 0");
        const DevRelease R = generate_release(b->terrain, *r, p->rho, b->stream);
        const int sid = batch_add_arrays(b, p, R.Np, R.x, R.v, R.vz, R.h, R.m, R.z);  // binning synchronises before R is freed
        if (sid_out) *sid_out = sid;
    });
}

slab_status slab_batch_run(slab_batch* b, int64_t max_steps, int64_t* steps_out) {
    if (!b) return SLAB_E_ARG;
    return bguard(b, [&] {
        bneed(b->E->nscn > 0, SLAB_E_STATE, "empty batch");
        run_t0(b);
        b->E->arm(max_steps, 0);
        int64_t done = 0;
        while (done < max_steps) {
            const int k = (int)std::min<int64_t>(b->chunk, max_steps - done);
            b->E->enqueue_steps(k);
            done += k;
            b->E->check_capacity();
            pull_all(b);
            bool all_stopped = true, gave_up = false;
            for (int s = 0; s < b->E->nscn; ++s) {
                all_stopped &= b->h_ctl[s].stop != 0;
                gave_up |= (b->h_ctl[s].err & ERR_TIMEOUT) != 0;
            }
            if (gave_up) {  // a persistent launch left its step half done: no step may follow
                b->E->dead = true;
                break;
            }
            if (all_stopped) break;
        }
        pull_all(b);
        raise_errors(b);
        if (steps_out) *steps_out = done;
    });
}

slab_status slab_batch_state(slab_batch* b, int32_t sid, double* time, int32_t* frame, int64_t* steps) {
    if (!b) return SLAB_E_ARG;
    return bguard(b, [&] {
        bneed(sid >= 0 && sid < b->E->nscn, SLAB_E_NOTFOUND, "unknown scenario");
        pull_all(b);
        if (time) *time = b->h_ctl[sid].time;
        if (frame) *frame = b->h_ctl[sid].frame;
        if (steps) *steps = b->h_ctl[sid].steps;
    });
}

slab_status slab_batch_scenario_status(slab_batch* b, int32_t sid) {
    if (!b) return SLAB_E_ARG;
    slab_status st = SLAB_OK;
    const slab_status g = bguard(b, [&] {
        bneed(sid >= 0 && sid < b->E->nscn, SLAB_E_NOTFOUND, "unknown scenario");
        pull_all(b);
        st = status_of(b->h_ctl[sid].err);
    });
    return g != SLAB_OK ? g : st;
}

slab_status slab_batch_download_particles(slab_batch* b, int32_t sid, double* x, double* v, double* vz, double* h, double* A, double* m,
                                          double* z) {
    if (!b) return SLAB_E_ARG;
    return bguard(b, [&] {
        bneed(sid >= 0 && sid < b->E->nscn, SLAB_E_NOTFOUND, "unknown scenario");
        b->E->download_particles(sid, x, v, vz, h, A, m, z, b->params[sid].rho);
    });
}

slab_status slab_batch_moments(slab_batch* b, int32_t sid, double out[6]) {
    if (!b || !out) return SLAB_E_ARG;
    return bguard(b, [&] {
        bneed(sid >= 0 && sid < b->E->nscn, SLAB_E_NOTFOUND, "unknown scenario");
        b->E->moments(sid, out);
    });
}

slab_status slab_batch_download_max(slab_batch* b, int32_t sid, double* h_max, double* v_max2) {
    if (!b) return SLAB_E_ARG;
    return bguard(b, [&] {
        bneed(sid >= 0 && sid < b->E->nscn, SLAB_E_NOTFOUND, "unknown scenario");
        b->E->download_max(sid, h_max, v_max2);
    });
}

slab_status slab_batch_download_max_box(slab_batch* b, int32_t sid, int32_t box[4], double* h_max, double* v_max2, int64_t cap_nodes) {
    if (!b || !box) return SLAB_E_ARG;
    return bguard(b, [&] {
        bneed(sid >= 0 && sid < b->E->nscn, SLAB_E_NOTFOUND, "unknown scenario");
        int bx[4];
        b->E->box_of_blocks(sid, bx);
        for (int k = 0; k < 4; ++k) box[k] = bx[k];
        const int64_t nI = bx[1] - bx[0] + 1, nJ = bx[3] - bx[2] + 1;
        if (!h_max || !v_max2 || nI <= 0 || nJ <= 0) return;
        bneed(nI * nJ <= cap_nodes, SLAB_E_ARG, "cap_nodes smaller than the box");
        b->E->download_max_box(sid, bx, h_max, v_max2);
    });
}

slab_status slab_batch_work_counters(slab_batch* b, int64_t out[2]) {
    if (!b || !out) return SLAB_E_ARG;
    return bguard(b, [&] {
        pull_all(b);
        out[0] = out[1] = 0;
        for (int s = 0; s < b->E->nscn; ++s) {
            out[0] += b->h_ctl[s].steps * (int64_t)b->Np[s];
            out[1] += (int64_t)b->h_ctl[s].node_steps;
        }
    });
}

slab_status slab_batch_set_stream(slab_batch* b, void* stream) {
    if (!b) return SLAB_E_ARG;
    return bguard(b, [&] {
        bneed(b->E->nscn == 0, SLAB_E_STATE, "set the stream before adding scenarios");
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : b->own_stream;
        b->E->st = s;
        b->stream = s;
    });
}

int32_t slab_batch_scenario_particles(const slab_batch* b, int32_t sid) {
    if (!b || sid < 0 || sid >= (int32_t)b->Np.size()) return -1;
    return b->Np[sid];
}

int64_t slab_batch_kernel_launches(const slab_batch* b) { return b && b->E ? b->E->nlaunch : 0; }

slab_status slab_batch_set_profiling(slab_batch* b, int32_t on) {
    if (!b) return SLAB_E_ARG;
    return bguard(b, [&] {
        b->E->timer.collect();
        b->E->timer.reset();
        b->E->timer.on = on != 0;
    });
}

slab_status slab_batch_phase_times(slab_batch* b, double out[5]) {
    if (!b || !out) return SLAB_E_ARG;
    return bguard(b, [&] {
        b->E->timer.collect();
        for (int k = 0; k < 5; ++k) out[k] = b->E->timer.acc[k];
    });
}

slab_status slab_batch_launch_shapes(slab_batch* b, int32_t out[6]) {
    if (!b || !out) return SLAB_E_ARG;
    return bguard(b, [&] {
        int g[5];
        b->E->launch_shapes(g);
        for (int k = 0; k < 5; ++k) out[k] = g[k];
        out[5] = b->E->tune.tunes;
    });
}

slab_status slab_batch_set_persistent(slab_batch* b, int32_t on, int64_t limit_cycles) {
    if (!b || limit_cycles < 0) return SLAB_E_ARG;
    return bguard(b, [&] { b->E->set_persistent(on != 0, limit_cycles); });
}

slab_status slab_batch_set_launch_shapes(slab_batch* b, const int32_t grids[5], int32_t tune) {
    if (!b) return SLAB_E_ARG;
    if (grids)
        for (int k = 0; k < 5; ++k)
            if (grids[k] < 0) return SLAB_E_ARG;
    return bguard(b, [&] { b->E->fix_shapes(grids, tune != 0); });
}

const char* slab_batch_last_error(const slab_batch* b) { return b ? b->err.c_str() : "null batch"; }

void slab_batch_destroy(slab_batch* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    b->E.reset();
    b->terrain.z.reset();
    b->terrain.grad.reset();
    b->terrain.cos_t.reset();
    b->terrain.dem32.reset();
    if (b->d_ctl) cudaFree(b->d_ctl);
    if (b->h_ctl) cudaFreeHost(b->h_ctl);
    if (b->own_stream) cudaStreamDestroy(b->own_stream);
    delete b;
}

}  // extern "C"
