// Serving: a request loop that admits scenario solves as they arrive and runs
// them with continuous batching on one GPU.
//
//  - slab_server_submit copies a scenario (parameters + particles) into a
//    queue and returns at once.
//  - A worker thread owns the GPU. Between chunks of batched steps it admits
//    queued requests into free scenario slots while their estimated HBM
//    footprint fits the budget, runs the t=0 pass of the new ones, advances
//    every running scenario by one chunk (one launch per kernel per step for
//    all of them, each with its own dt and friction), and retires the ones
//    that reached their total_time: results go to host memory and the slot's
//    memory and node blocks return to the pools.
//  - Particle and grid state stay on the device from admission to
//    retirement. Time to result is measured from submission.
// A request's result is bitwise the same as running it alone (FP32 split):
// nothing a kernel sums mixes scenarios and every sum is exact or in a fixed
// order.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "engine.hpp"
#include "engine32.hpp"
#include "release.hpp"

namespace slab {
void set_thread_error(const std::string& msg);
}

using namespace slab;

namespace {

using clk = std::chrono::steady_clock;

enum { REQ_QUEUED = SLAB_REQ_QUEUED, REQ_RUNNING = SLAB_REQ_RUNNING, REQ_DONE = SLAB_REQ_DONE, REQ_CANCELLED = SLAB_REQ_CANCELLED, REQ_FAILED = SLAB_REQ_FAILED };

struct Request {
    int64_t id = 0;
    slab_params p{};
    int Np = 0;
    std::vector<double> x, v, vz, h, m, z;
    bool has_release = false;  // particles built on the device at admission (slab_server_submit_release)
    slab_release rel{};
    int state = REQ_QUEUED;
    bool cancel = false;
    int slot = -1;
    int64_t footprint = 0;
    clk::time_point t_submit, t_start, t_done;
    int64_t steps = 0;
    double sim_time = 0;
    int box[4] = {0, -1, 0, -1};
    std::vector<double> hmax, vmax2;
    std::vector<double> px, pv, ph, pm;
    std::string err;
};

}  // namespace

struct slab_server {
    Terrain terrain;
    cudaStream_t stream = nullptr;
    int max_slots = 0;
    int chunk = 32;
    Ctl* d_ctl = nullptr;
    Ctl* h_ctl = nullptr;
    std::unique_ptr<Engine32> E;
    int64_t budget = 0, used = 0;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<int64_t> queue;
    std::map<int64_t, Request> reqs;
    std::vector<int64_t> slot_req;
    int64_t next_id = 1;
    int admitting = 0;  // taken from the queue, not yet in a slot
    bool stopping = false;
    std::thread worker;
    std::string err;
    // statistics
    int64_t completed = 0, batched_steps = 0, particle_steps = 0;
    std::vector<double> ttr;  // seconds to result of completed requests
    clk::time_point t_first_submit, t_last_done;
    bool any_submit = false;
    double busy_s = 0;
    // where the worker's time goes
    double admit_s = 0, chunk_s = 0, retire_s = 0;
    int64_t chunks = 0, running_sum = 0, running_max = 0, grown = 0;
};

namespace {

int64_t footprint_of(const slab_server* s, int Np) {
    const int64_t TX = (s->terrain.Nx + TILE - 1) / TILE, TY = (s->terrain.Ny + TILE - 1) / TILE, nt = TX * TY;
    const int64_t act = std::min<int64_t>(nt, Np / 4 + 256);
    // particle buffers, tile metadata, work descriptors and partials, node blocks
    return (int64_t)Np * 80 + nt * (2 * GRP_STRIDE * 4 + 7 * 4) + act * (PART_STRIDE * 4 + (int64_t)sizeof(TileDesc) + 8) +
           act * NCELL * 36;
}

Ctl empty_ctl(const slab_server* s) {
    Ctl c;
    std::memset(&c, 0, sizeof(Ctl));
    c.dx = s->terrain.dx;
    c.one_over_dx = 1. / s->terrain.dx;
    c.total_time = -1.0;  // never runs
    c.stop = 1;
    return c;
}

void finish(slab_server* s, int slot, int state, const std::string& err) {
    std::unique_lock<std::mutex> lk(s->mu);
    Request& r = s->reqs[s->slot_req[slot]];
    lk.unlock();
    if (state == REQ_DONE) {
        s->E->box_of_blocks(slot, r.box);
        const int nI = r.box[1] - r.box[0] + 1, nJ = r.box[3] - r.box[2] + 1;
        if (nI > 0 && nJ > 0) {
            r.hmax.resize((size_t)nI * nJ);
            r.vmax2.resize((size_t)nI * nJ);
            s->E->download_max_box(slot, r.box, r.hmax.data(), r.vmax2.data());
        }
        r.px.resize(2 * (size_t)r.Np);
        r.pv.resize(2 * (size_t)r.Np);
        r.ph.resize(r.Np);
        r.pm.resize(r.Np);
        s->E->download_particles(slot, r.px.data(), r.pv.data(), nullptr, r.ph.data(), nullptr, r.pm.data(), nullptr, r.p.rho);
    }
    s->E->retire(slot, empty_ctl(s));
    lk.lock();
    r.state = state;
    r.err = err;
    r.t_done = clk::now();
    r.slot = -1;
    s->used -= r.footprint;
    s->slot_req[slot] = -1;
    if (state == REQ_DONE) {
        s->completed += 1;
        s->ttr.push_back(std::chrono::duration<double>(r.t_done - r.t_submit).count());
        s->t_last_done = r.t_done;
    }
    std::vector<double>().swap(r.x);
    std::vector<double>().swap(r.v);
    std::vector<double>().swap(r.vz);
    std::vector<double>().swap(r.h);
    std::vector<double>().swap(r.m);
    std::vector<double>().swap(r.z);
    s->cv.notify_all();
}

void worker_loop(slab_server* s) {
    for (;;) {
        // ---- admission (requests that fit a free slot and the memory budget)
        std::vector<int64_t> admit;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            bool running = false;
            for (int64_t r : s->slot_req) running |= r >= 0;
            if (!running && s->queue.empty()) {
                if (s->stopping) return;
                s->cv.wait_for(lk, std::chrono::milliseconds(20));
                continue;
            }
            if (s->stopping) return;
            int free_slots = 0;
            for (int64_t r : s->slot_req) free_slots += r < 0;
            int64_t used = s->used;
            while (!s->queue.empty() && free_slots > 0) {
                Request& r = s->reqs[s->queue.front()];
                if (r.cancel) {
                    r.state = REQ_CANCELLED;
                    s->queue.pop_front();
                    continue;
                }
                if (used + r.footprint > s->budget && (used > 0 || !admit.empty())) break;  // wait for memory
                used += r.footprint;
                admit.push_back(r.id);
                s->queue.pop_front();
                --free_slots;
            }
            s->admitting += (int)admit.size();
        }
        const auto t0 = clk::now();
        bool new_ones = false;
        auto secs = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };
        for (int64_t id : admit) {
            Request* r;
            {
                std::lock_guard<std::mutex> lk(s->mu);
                r = &s->reqs[id];
            }
            try {
                int slot = -1;
                for (int k = 0; k < s->max_slots; ++k)
                    if (s->slot_req[k] < 0) {
                        slot = k;
                        break;
                    }
                Ctl& c = s->h_ctl[slot];
                std::memset(&c, 0, sizeof(Ctl));
                c.dx = s->terrain.dx;
                c.one_over_dx = 1. / s->terrain.dx;
                c.C_cfl = r->p.C_cfl;
                c.dt_max = r->p.dt_max;
                c.output_dt = r->p.output_dt;
                c.total_time = r->p.total_time;
                c.stop = 1;
                int got;
                if (r->has_release) {  // the release's particles, built on the device
                    const DevRelease R = generate_release(s->terrain, r->rel, r->p.rho, s->stream);
                    r->Np = R.Np;
                    got = s->E->add_scenario(r->p, s->d_ctl + slot, &c, R.Np, R.x, R.v, R.vz, R.h, R.m, R.z, slot);
                } else {
                    got = s->E->add_scenario(r->p, s->d_ctl + slot, &c, r->Np, r->x.data(), r->v.data(), r->vz.data(), r->h.data(),
                                             r->m.data(), r->z.data(), slot);
                }
                std::lock_guard<std::mutex> lk(s->mu);
                s->slot_req[got] = id;
                r->slot = got;
                r->state = REQ_RUNNING;
                r->t_start = clk::now();
                s->used += r->footprint;
                s->admitting -= 1;
                new_ones = true;
            } catch (const Error& e) {
                std::lock_guard<std::mutex> lk(s->mu);
                r->state = REQ_FAILED;
                r->err = e.msg;
                r->t_done = clk::now();
                s->admitting -= 1;
                s->cv.notify_all();
            }
        }
        try {
            const auto t1 = clk::now();
            s->admit_s += secs(t0, t1);
            if (new_ones) s->E->launch_t0();
            // ---- one chunk of batched steps for every running scenario
            s->E->arm(s->chunk, 0);
            s->E->enqueue_steps(s->chunk);
            if (s->E->check_capacity()) s->grown += 1;
            const int n = s->E->nscn;
            SLAB_CUDA(cudaMemcpyAsync(s->h_ctl, s->d_ctl, n * sizeof(Ctl), cudaMemcpyDeviceToHost, s->stream));
            SLAB_CUDA(cudaStreamSynchronize(s->stream));
            const auto t2 = clk::now();
            s->chunk_s += secs(t1, t2);
            s->batched_steps += s->chunk;
            {
                int running = 0;
                std::lock_guard<std::mutex> lk(s->mu);
                for (int64_t r : s->slot_req) running += r >= 0;
                s->chunks += 1;
                s->running_sum += running;
                s->running_max = std::max<int64_t>(s->running_max, running);
            }
            // ---- retire finished / failed / cancelled scenarios
            for (int k = 0; k < n; ++k) {
                int64_t id;
                bool cancel;
                {
                    std::lock_guard<std::mutex> lk(s->mu);
                    id = s->slot_req[k];
                    if (id < 0) continue;
                    cancel = s->reqs[id].cancel;
                }
                const Ctl& c = s->h_ctl[k];
                if (c.err & ERR_TIMEOUT)  // a persistent launch gave up at a barrier: the engine's step state is incomplete
                    throw Error{SLAB_E_TIMEOUT, "a bounded device wait gave up; the engine stopped"};
                if (c.err) {
                    finish(s, k, REQ_FAILED, "device error flags " + std::to_string(c.err));
                } else if (cancel) {
                    finish(s, k, REQ_CANCELLED, "");
                } else if (c.stop && !(c.time < c.total_time)) {
                    {
                        std::lock_guard<std::mutex> lk(s->mu);
                        Request& r = s->reqs[id];
                        r.steps = c.steps;
                        r.sim_time = c.time;
                        s->particle_steps += c.steps * (int64_t)r.Np;
                    }
                    finish(s, k, REQ_DONE, "");
                }
            }
            s->retire_s += secs(t2, clk::now());
        } catch (const Error& e) {
            std::lock_guard<std::mutex> lk(s->mu);
            s->err = e.msg;
            for (int k = 0; k < s->max_slots; ++k)
                if (s->slot_req[k] >= 0) {
                    s->reqs[s->slot_req[k]].state = REQ_FAILED;
                    s->reqs[s->slot_req[k]].err = e.msg;
                    s->slot_req[k] = -1;
                }
            s->stopping = true;
            s->cv.notify_all();
            return;
        }
        s->busy_s += std::chrono::duration<double>(clk::now() - t0).count();
    }
}

template <typename F> slab_status sguard(slab_server* s, F&& f) {
    try {
        f();
        return SLAB_OK;
    } catch (const Error& e) {
        if (s) s->err = e.msg;
        set_thread_error(e.msg);
        return e.code;
    } catch (const std::exception& e) {
        if (s) s->err = e.what();
        set_thread_error(e.what());
        return SLAB_E_ARG;
    }
}

void sneed(bool ok, slab_status code, const char* msg) {
    if (!ok) throw Error{code, msg};
}

double quantile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (v.size() - 1);
    const size_t i = (size_t)pos;
    const double f = pos - i;
    return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
}

}  // namespace

extern "C" {

slab_status slab_server_create(const slab_terrain_desc* td, const double* z, const slab_server_config* cfg, slab_server** out) {
    if (!td || !z || !out || !cfg) return SLAB_E_ARG;
    *out = nullptr;
    slab_server* s = new slab_server();
    slab_status st = sguard(s, [&] {
        sneed(cfg->max_scenarios > 0, SLAB_E_ARG, "max_scenarios must be > 0");
        sneed(td->Nx >= 4 && td->Ny >= 4 && td->dx > 0, SLAB_E_ARG, "invalid terrain");
        SLAB_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
        s->max_slots = cfg->max_scenarios;
        s->chunk = cfg->chunk_steps > 0 ? cfg->chunk_steps : 32;
        s->d_ctl = dmalloc<Ctl>(s->max_slots);
        SLAB_CUDA(cudaMallocHost(&s->h_ctl, s->max_slots * sizeof(Ctl)));
        Terrain& t = s->terrain;
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
        SLAB_CUDA(cudaMemcpyAsync(t.z.get(), z, n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
        compute_terrain_metrics(t, s->stream);
        const int64_t ntiles = (int64_t)((t.Nx + TILE - 1) / TILE) * ((t.Ny + TILE - 1) / TILE);
        s->E.reset(new Engine32(t, s->stream, s->max_slots, std::min<int64_t>(ntiles, 1 << 16), true));
        const Ctl e = empty_ctl(s);
        for (int k = 0; k < s->max_slots; ++k) s->h_ctl[k] = e;
        SLAB_CUDA(cudaMemcpyAsync(s->d_ctl, s->h_ctl, s->max_slots * sizeof(Ctl), cudaMemcpyHostToDevice, s->stream));
        SLAB_CUDA(cudaStreamSynchronize(s->stream));
        size_t free_b = 0, total_b = 0;
        SLAB_CUDA(cudaMemGetInfo(&free_b, &total_b));
        s->budget = cfg->hbm_budget_bytes > 0 ? cfg->hbm_budget_bytes : (int64_t)(free_b / 2);
        s->slot_req.assign(s->max_slots, -1);
        s->worker = std::thread(worker_loop, s);
    });
    if (st != SLAB_OK) {
        slab_server_destroy(s);
        return st;
    }
    *out = s;
    return SLAB_OK;
}

slab_status slab_server_submit(slab_server* s, const slab_params* p, int32_t Np, const double* x, const double* v, const double* vz,
                               const double* h, const double* A, const double* m, const double* z, int64_t* request_id) {
    if (!s || !p || !request_id) return SLAB_E_ARG;
    (void)A;
    return sguard(s, [&] {
        sneed(Np > 0 && x && v && vz && h && m && z, SLAB_E_ARG, "invalid particle arrays");
        sneed(p->precision == SLAB_FP32_SPLIT, SLAB_E_ARG, "the server runs the FP32_SPLIT arithmetic");
        sneed(p->total_time >= 0 && p->dt_max > 0 && p->output_dt > 0 && p->C_cfl > 0, SLAB_E_ARG, "invalid parameters");
        Request r;
        r.p = *p;
        r.Np = Np;
        r.x.assign(x, x + 2 * (size_t)Np);
        r.v.assign(v, v + 2 * (size_t)Np);
        r.vz.assign(vz, vz + Np);
        r.h.assign(h, h + Np);
        r.m.assign(m, m + Np);
        r.z.assign(z, z + Np);
        r.footprint = footprint_of(s, Np);
        r.t_submit = clk::now();
        std::lock_guard<std::mutex> lk(s->mu);
        sneed(!s->stopping, SLAB_E_STATE, "server is shutting down");
        r.id = s->next_id++;
        if (!s->any_submit) {
            s->any_submit = true;
            s->t_first_submit = r.t_submit;
        }
        *request_id = r.id;
        s->queue.push_back(r.id);
        s->reqs.emplace(r.id, std::move(r));
        s->cv.notify_all();
    });
}

slab_status slab_server_submit_release(slab_server* s, const slab_params* p, const slab_release* rel, int64_t* request_id) {
    if (!s || !p || !rel || !request_id) return SLAB_E_ARG;
    return sguard(s, [&] {
        sneed(p->precision == SLAB_FP32_SPLIT, SLAB_E_ARG, "the server runs the FP32_SPLIT arithmetic");
        sneed(p->total_time >= 0 && p->dt_max > 0 && p->output_dt > 0 && p->C_cfl > 0 && p->rho > 0, SLAB_E_ARG, "invalid parameters");
        sneed(rel->a > 0 && rel->b > 0 && rel->h0 > 0 && (rel->type == SLAB_RELEASE_RECTANGLE || rel->type == SLAB_RELEASE_ELLIPSE), SLAB_E_ARG,
              "invalid release");
        Request r;
        r.p = *p;
        r.has_release = true;
        r.rel = *rel;
        const int64_t est = release_estimate(*rel, s->terrain.dx);
        sneed(est < INT32_MAX, SLAB_E_ARG, "release too large");
        r.Np = (int)est;  // until admission builds the particles
        r.footprint = footprint_of(s, (int)est);
        r.t_submit = clk::now();
        std::lock_guard<std::mutex> lk(s->mu);
        sneed(!s->stopping, SLAB_E_STATE, "server is shutting down");
        r.id = s->next_id++;
        if (!s->any_submit) {
            s->any_submit = true;
            s->t_first_submit = r.t_submit;
        }
        *request_id = r.id;
        s->queue.push_back(r.id);
        s->reqs.emplace(r.id, std::move(r));
        s->cv.notify_all();
    });
}

slab_status slab_server_particles(slab_server* s, int64_t id, int32_t* Np) {
    if (!s || !Np) return SLAB_E_ARG;
    return sguard(s, [&] {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->reqs.find(id);
        sneed(it != s->reqs.end(), SLAB_E_NOTFOUND, "unknown request");
        sneed(it->second.state != REQ_QUEUED || !it->second.has_release, SLAB_E_STATE, "the release has not been built yet");
        *Np = it->second.Np;
    });
}

slab_status slab_server_poll(slab_server* s, int64_t id, int32_t* state, double* seconds_to_result) {
    if (!s) return SLAB_E_ARG;
    return sguard(s, [&] {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->reqs.find(id);
        sneed(it != s->reqs.end(), SLAB_E_NOTFOUND, "unknown request");
        if (state) *state = it->second.state;
        if (seconds_to_result)
            *seconds_to_result = it->second.state >= REQ_DONE ? std::chrono::duration<double>(it->second.t_done - it->second.t_submit).count() : -1.0;
    });
}

slab_status slab_server_wait(slab_server* s, int64_t id, double timeout_s) {
    if (!s) return SLAB_E_ARG;
    return sguard(s, [&] {
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->reqs.find(id);
        sneed(it != s->reqs.end(), SLAB_E_NOTFOUND, "unknown request");
        const bool ok = s->cv.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                       [&] { return s->reqs[id].state >= REQ_DONE || s->stopping; });
        sneed(ok, SLAB_E_TIMEOUT, "request not finished in time");
        sneed(s->reqs[id].state == REQ_DONE, s->reqs[id].state == REQ_CANCELLED ? SLAB_E_STATE : SLAB_E_CUDA,
              s->reqs[id].state == REQ_CANCELLED ? "request cancelled" : "request failed");
    });
}

slab_status slab_server_result(slab_server* s, int64_t id, int32_t box[4], double* h_max, double* v_max2, int64_t cap_nodes,
                               double* x_xy, double* v_xy, double* h, double* mass, double* info) {
    if (!s) return SLAB_E_ARG;
    return sguard(s, [&] {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->reqs.find(id);
        sneed(it != s->reqs.end(), SLAB_E_NOTFOUND, "unknown request");
        const Request& r = it->second;
        sneed(r.state == REQ_DONE, SLAB_E_STATE, "request has no result");
        if (box) std::memcpy(box, r.box, sizeof(r.box));
        const int64_t n = (int64_t)r.hmax.size();
        if (h_max || v_max2) sneed(cap_nodes >= n, SLAB_E_ARG, "max-map capacity too small");
        if (h_max) std::copy(r.hmax.begin(), r.hmax.end(), h_max);
        if (v_max2) std::copy(r.vmax2.begin(), r.vmax2.end(), v_max2);
        if (x_xy) std::copy(r.px.begin(), r.px.end(), x_xy);
        if (v_xy) std::copy(r.pv.begin(), r.pv.end(), v_xy);
        if (h) std::copy(r.ph.begin(), r.ph.end(), h);
        if (mass) std::copy(r.pm.begin(), r.pm.end(), mass);
        if (info) {
            info[0] = (double)r.steps;
            info[1] = r.sim_time;
            info[2] = std::chrono::duration<double>(r.t_done - r.t_submit).count();
            info[3] = std::chrono::duration<double>(r.t_start - r.t_submit).count();
        }
    });
}

slab_status slab_server_cancel(slab_server* s, int64_t id) {
    if (!s) return SLAB_E_ARG;
    return sguard(s, [&] {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->reqs.find(id);
        sneed(it != s->reqs.end(), SLAB_E_NOTFOUND, "unknown request");
        it->second.cancel = true;
        if (it->second.state == REQ_QUEUED) {
            it->second.state = REQ_CANCELLED;
            s->queue.erase(std::remove(s->queue.begin(), s->queue.end(), id), s->queue.end());
        }
        s->cv.notify_all();
    });
}

slab_status slab_server_drain(slab_server* s, double timeout_s) {
    if (!s) return SLAB_E_ARG;
    return sguard(s, [&] {
        std::unique_lock<std::mutex> lk(s->mu);
        const bool ok = s->cv.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] {
            if (s->stopping) return true;
            if (!s->queue.empty() || s->admitting) return false;
            for (int64_t r : s->slot_req)
                if (r >= 0) return false;
            return true;
        });
        sneed(ok, SLAB_E_TIMEOUT, "requests still running");
        sneed(s->err.empty(), SLAB_E_CUDA, "server stopped after an error");
    });
}

slab_status slab_server_stats(slab_server* s, double out[8]) {
    if (!s || !out) return SLAB_E_ARG;
    return sguard(s, [&] {
        std::lock_guard<std::mutex> lk(s->mu);
        out[0] = (double)s->completed;
        out[1] = quantile(s->ttr, 0.5);
        out[2] = quantile(s->ttr, 0.99);
        const double span = s->completed ? std::chrono::duration<double>(s->t_last_done - s->t_first_submit).count() : 0.0;
        out[3] = span > 0 ? s->completed / span : 0.0;
        out[4] = (double)s->particle_steps;
        out[5] = (double)s->batched_steps;
        out[6] = s->busy_s;
        out[7] = (double)s->used;
    });
}

slab_status slab_server_timing(slab_server* s, double out[8]) {
    if (!s || !out) return SLAB_E_ARG;
    return sguard(s, [&] {
        std::lock_guard<std::mutex> lk(s->mu);
        out[0] = s->admit_s;
        out[1] = s->chunk_s;
        out[2] = s->retire_s;
        out[3] = (double)s->chunks;
        out[4] = s->chunks ? (double)s->running_sum / (double)s->chunks : 0.0;
        out[5] = (double)s->running_max;
        out[6] = (double)s->grown;
        out[7] = (double)s->E->nlaunch;
    });
}

const char* slab_server_last_error(const slab_server* s) { return s ? s->err.c_str() : "null server"; }

void slab_server_destroy(slab_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
        s->cv.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    if (s->stream) cudaStreamSynchronize(s->stream);
    s->E.reset();
    s->terrain.z.reset();
    s->terrain.grad.reset();
    s->terrain.cos_t.reset();
    s->terrain.dem32.reset();
    if (s->d_ctl) cudaFree(s->d_ctl);
    if (s->h_ctl) cudaFreeHost(s->h_ctl);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

}  // extern "C"
