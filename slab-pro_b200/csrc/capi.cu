// The C ABI of libslab_gpu.so (include/slab_gpu.h): context management,
// argument checks, the host side of the step loop (arming the device control
// block, replaying step graphs until a frame), and error translation.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <string>

#include "engine.hpp"
#include "release.hpp"

using namespace slab;

namespace slab {
// message of the last failed context-free call on this thread (slab_last_error(NULL))
static thread_local std::string t_last_error;
void set_thread_error(const std::string& msg) { t_last_error = msg; }
}  // namespace slab

// One output frame in flight (slab_frame_capture / slab_frame_wait): the
// packed frame on the device, its pinned host copy, and the event that marks
// the end of the copy.
struct FrameSlot {
    dptr<float> dev;
    float* host = nullptr;  // pinned
    size_t cap = 0;         // floats in both buffers
    cudaEvent_t packed = nullptr, copied = nullptr;
    bool pending = false;   // a copy was started and not yet waited for
    slab_frame meta{};
};

struct slab_ctx {
    Terrain terrain;
    slab_params params{};
    bool have_params = false;
    bool uploaded = false;
    bool initial_done = false;
    int Np = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    int device = 0;
    Ctl* d_ctl = nullptr;
    Ctl* h_ctl = nullptr;  // pinned mirror
    std::unique_ptr<Path> path;
    std::string err;
    int64_t extra_launches = 0;
    int chunk = 32;
    int persist = -1;              // -1: the engine's default; 0 / 1 set by slab_set_persistent
    long long persist_limit = 0;
    cudaStream_t copy_stream = nullptr;  // frame copies to the host
    FrameSlot frames[2];
};

namespace {

__global__ void k_arm(Ctl* c, int64_t steps_left, int32_t stop_at_frame) {
    if (threadIdx.x == 0) {
        c->stop = 0;
        c->frame_hit = 0;
        c->steps_left = steps_left;
        c->stop_at_frame = stop_at_frame;
    }
}

template <typename F> slab_status guard(slab_ctx* ctx, F&& f) {
    try {
        f();
        if (ctx) ctx->err.clear();
        return SLAB_OK;
    } catch (const Error& e) {
        if (ctx) ctx->err = e.msg;
        return e.code;
    } catch (const std::bad_alloc&) {
        if (ctx) ctx->err = "host allocation failed";
        return SLAB_E_OOM;
    } catch (const std::exception& e) {
        if (ctx) ctx->err = e.what();
        return SLAB_E_ARG;
    }
}

void need(bool ok, slab_status code, const char* msg) {
    if (!ok) throw Error{code, msg};
}

void check_params(const slab_params& p) {
    need(std::isfinite(p.gravity) && p.gravity > 0, SLAB_E_ARG, "gravity must be > 0");
    need(std::isfinite(p.rho) && p.rho > 0, SLAB_E_ARG, "rho must be > 0");
    need(std::isfinite(p.C_cfl) && p.C_cfl > 0, SLAB_E_ARG, "C_cfl must be > 0");
    need(std::isfinite(p.dt_max) && p.dt_max > 0, SLAB_E_ARG, "dt_max must be > 0");
    need(std::isfinite(p.flip_ratio) && p.flip_ratio >= 0 && p.flip_ratio <= 1, SLAB_E_ARG, "flip_ratio must be in [0,1]");
    need(std::isfinite(p.output_dt) && p.output_dt > 0, SLAB_E_ARG, "output_dt must be > 0");
    need(std::isfinite(p.total_time) && p.total_time >= 0, SLAB_E_ARG, "total_time must be >= 0");
    need(p.friction.type >= SLAB_COULOMB && p.friction.type <= SLAB_MU_I, SLAB_E_ARG, "unknown friction type");
    need(p.precision == SLAB_FP64_PLAIN || p.precision == SLAB_FP32_SPLIT, SLAB_E_ARG, "unknown precision");
    if (p.friction.type == SLAB_VOELLMY) need(p.friction.voellmy_xi > 0, SLAB_E_ARG, "voellmy xi must be > 0");
    if (p.friction.type == SLAB_MU_I) need(p.friction.I0 > 0 && p.friction.phi > 0, SLAB_E_ARG, "mu_I needs I0 > 0 and phi > 0");
}

void reset_ctl(slab_ctx* c) {
    Ctl& h = *c->h_ctl;
    std::memset(&h, 0, sizeof(Ctl));
    h.dx = c->terrain.dx;
    h.one_over_dx = 1. / c->terrain.dx;
    h.C_cfl = c->params.C_cfl;
    h.dt_max = c->params.dt_max;
    h.output_dt = c->params.output_dt;
    h.total_time = c->params.total_time;
    h.stop = 1;
    h.pos_acc[0] = 0x7ff0000000000000ull;
    h.pos_acc[2] = 0x7ff0000000000000ull;
    SLAB_CUDA(cudaMemcpyAsync(c->d_ctl, &h, sizeof(Ctl), cudaMemcpyHostToDevice, c->stream));
    SLAB_CUDA(cudaStreamSynchronize(c->stream));
}

void pull_ctl(slab_ctx* c) {
    SLAB_CUDA(cudaMemcpyAsync(c->h_ctl, c->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c->stream));
    SLAB_CUDA(cudaStreamSynchronize(c->stream));
}

void raise_device_errors(slab_ctx* c) {
    const int e = c->h_ctl->err;
    if (e & ERR_NONFINITE) throw Error{SLAB_E_NONFINITE, "non-finite particle state"};
    if (e & (ERR_DOMAIN | ERR_MOVE)) throw Error{SLAB_E_DOMAIN, "a particle stencil left the terrain"};
    if (e & ERR_CAPACITY) throw Error{SLAB_E_OOM, "device capacity exceeded"};
    if (e & ERR_TIMEOUT) throw Error{SLAB_E_TIMEOUT, "bounded device wait gave up"};  // the engine takes no further steps
}

void arm(slab_ctx* c, int64_t steps_left, int stop_at_frame) {
    if (c->path->arm(steps_left, stop_at_frame)) return;
    k_arm<<<1, 32, 0, c->stream>>>(c->d_ctl, steps_left, stop_at_frame);
    SLAB_CUDA(cudaGetLastError());
    ++c->extra_launches;
}

void enqueue_nsteps(slab_ctx* c, int64_t nsteps) {
    arm(c, nsteps, 0);
    int64_t k = 0;
    for (; k + c->chunk <= nsteps; k += c->chunk) c->path->enqueue_steps(c->chunk);
    if (k < nsteps) c->path->enqueue_steps((int)(nsteps - k));
}

void advance(slab_ctx* c, int64_t nsteps, bool stop_at_frame, int64_t* steps_out) {
    need(c->uploaded, SLAB_E_STATE, "no particles uploaded");
    need(c->initial_done, SLAB_E_STATE, "call slab_initial_pass before advancing");
    pull_ctl(c);
    const int64_t s0 = c->h_ctl->steps;
    if (!stop_at_frame) {
        // the step budget is on the device; enqueue up to 8 chunks, then look
        // at the control block, so a run that stops at total_time long before
        // the budget does not keep the host enqueueing empty steps
        arm(c, nsteps, 0);
        const int64_t poll = 8 * (int64_t)c->chunk;
        int64_t k = 0;
        while (k < nsteps) {
            const int64_t end = std::min(nsteps, k + poll);
            for (; k + c->chunk <= end; k += c->chunk) c->path->enqueue_steps(c->chunk);
            if (k < end) {
                c->path->enqueue_steps((int)(end - k));
                k = end;
            }
            pull_ctl(c);
            if (c->h_ctl->stop || c->h_ctl->err) break;
        }
    } else {
        arm(c, nsteps, 1);
        double last_time = c->h_ctl->time;
        int stalled = 0;
        for (;;) {
            c->path->enqueue_steps(c->chunk);
            pull_ctl(c);
            if (c->h_ctl->stop) break;
            // dt > 0 always moves time forward; a chunk without progress
            // means the control block is stuck, so give up instead of spinning
            stalled = (c->h_ctl->time == last_time) ? stalled + 1 : 0;
            last_time = c->h_ctl->time;
            if (stalled > 4) throw Error{SLAB_E_TIMEOUT, "time does not advance"};
        }
    }
    raise_device_errors(c);
    if (steps_out) *steps_out = c->h_ctl->steps - s0;
}

}  // namespace

extern "C" {

const char* slab_version(void) { return "slab-b200 0.1 (sm_100a)"; }

const char* slab_status_name(slab_status s) {
    switch (s) {
        case SLAB_OK: return "SLAB_OK";
        case SLAB_E_ARG: return "SLAB_E_ARG";
        case SLAB_E_CUDA: return "SLAB_E_CUDA";
        case SLAB_E_OOM: return "SLAB_E_OOM";
        case SLAB_E_DOMAIN: return "SLAB_E_DOMAIN";
        case SLAB_E_NONFINITE: return "SLAB_E_NONFINITE";
        case SLAB_E_TIMEOUT: return "SLAB_E_TIMEOUT";
        case SLAB_E_STATE: return "SLAB_E_STATE";
        case SLAB_E_NOTFOUND: return "SLAB_E_NOTFOUND";
    }
    return "SLAB_E_UNKNOWN";
}

slab_status slab_create(const slab_terrain_desc* td, const double* z, slab_ctx** out) {
    if (!td || !z || !out) {
        set_thread_error("slab_create: terrain, z and out must not be NULL");
        return SLAB_E_ARG;
    }
    *out = nullptr;
    slab_ctx* c = new slab_ctx();
    slab_status s = guard(c, [&] {
        need(td->Nx >= 4 && td->Ny >= 4, SLAB_E_ARG, "terrain needs at least 4x4 nodes");
        need((int64_t)td->Nx * td->Ny < (int64_t(1) << 31), SLAB_E_ARG, "terrain too large (Nx*Ny must fit int32)");
        need(std::isfinite(td->dx) && td->dx > 0, SLAB_E_ARG, "dx must be > 0");
        SLAB_CUDA(cudaGetDevice(&c->device));
        SLAB_CUDA(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
        c->stream = c->own_stream;
        c->d_ctl = dmalloc<Ctl>(1);
        SLAB_CUDA(cudaMallocHost(&c->h_ctl, sizeof(Ctl)));
        Terrain& t = c->terrain;
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
        SLAB_CUDA(cudaMemcpyAsync(t.z.get(), z, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        compute_terrain_metrics(t, c->stream);
        ++c->extra_launches;
        SLAB_CUDA(cudaStreamSynchronize(c->stream));
    });
    if (s != SLAB_OK) {
        set_thread_error(c->err);  // the context goes: slab_last_error(NULL) keeps the message
        slab_destroy(c);
        return s;
    }
    *out = c;
    return SLAB_OK;
}

slab_status slab_set_params(slab_ctx* c, const slab_params* p) {
    if (!c || !p) return SLAB_E_ARG;
    return guard(c, [&] {
        check_params(*p);
        c->params = *p;
        c->have_params = true;
        c->uploaded = false;
        c->path.reset();
    });
}

slab_status slab_set_stream(slab_ctx* c, void* s) {
    if (!c) return SLAB_E_ARG;
    return guard(c, [&] {
        need(!c->path, SLAB_E_STATE, "set the stream before uploading particles");
        c->stream = s ? static_cast<cudaStream_t>(s) : c->own_stream;
    });
}

namespace {
// a new path over the context's terrain with these particles (host or device arrays)
void upload_arrays(slab_ctx* c, int32_t Np, const double* x, const double* v, const double* vz, const double* h, const double* A,
                   const double* m, const double* z) {
    c->uploaded = false;
    c->path.reset();
    reset_ctl(c);
    if (c->params.precision == SLAB_FP64_PLAIN)
        c->path = make_plain64(c->terrain, c->params, c->stream, c->d_ctl, c->h_ctl);
    else
        c->path = make_split32(c->terrain, c->params, c->stream, c->d_ctl, c->h_ctl);
    if (c->persist >= 0 && c->params.precision != SLAB_FP64_PLAIN) c->path->set_persistent(c->persist != 0, c->persist_limit);
    c->path->upload(Np, x, v, vz, h, A, m, z);
    pull_ctl(c);
    raise_device_errors(c);
    c->Np = Np;
    c->uploaded = true;
    c->initial_done = false;
}
}  // namespace

slab_status slab_upload_particles(slab_ctx* c, int32_t Np, const double* x, const double* v, const double* vz, const double* h,
                                  const double* A, const double* m, const double* z) {
    if (!c) return SLAB_E_ARG;
    return guard(c, [&] {
        need(c->have_params, SLAB_E_STATE, "slab_set_params first");
        need(Np > 0, SLAB_E_ARG, "Np must be > 0");
        need(x && v && vz && h && A && m && z, SLAB_E_ARG, "null particle array");
        std::atomic<int> bad_x{0}, bad_hm{0};
        parallel_ranges(Np, [&](int64_t b, int64_t e) {
            bool fx = false, fhm = false;
            for (int64_t q = b; q < e; ++q) {
                fx |= !(std::isfinite(x[2 * q]) && std::isfinite(x[2 * q + 1]));
                fhm |= !(h[q] > 0 && m[q] > 0);
            }
            if (fx) bad_x = 1;
            if (fhm) bad_hm = 1;
        });
        need(!bad_x, SLAB_E_ARG, "non-finite particle position");
        need(!bad_hm, SLAB_E_ARG, "particle h and mass must be > 0");
        upload_arrays(c, Np, x, v, vz, h, A, m, z);
    });
}

slab_status slab_upload_release(slab_ctx* c, const slab_release* r, int32_t* Np_out) {
    if (!c || !r) return SLAB_E_ARG;
    return guard(c, [&] {
        need(c->have_params, SLAB_E_STATE, "slab_set_params first");
        const DevRelease R = generate_release(c->terrain, *r, c->params.rho, c->stream);
        upload_arrays(c, R.Np, R.x, R.v, R.vz, R.h, R.A, R.m, R.z);  // synchronises before R is freed
        if (Np_out) *Np_out = R.Np;
    });
}

slab_status slab_initial_pass(slab_ctx* c) {
    if (!c) return SLAB_E_ARG;
    return guard(c, [&] {
        need(c->uploaded, SLAB_E_STATE, "no particles uploaded");
        c->path->initial_pass();
        pull_ctl(c);
        raise_device_errors(c);
        c->initial_done = true;
    });
}

slab_status slab_advance_to_frame(slab_ctx* c, double* time_out, int32_t* frame_out, int64_t* steps_out) {
    if (!c) return SLAB_E_ARG;
    return guard(c, [&] {
        advance(c, int64_t(1) << 62, true, steps_out);
        if (time_out) *time_out = c->h_ctl->time;
        if (frame_out) *frame_out = c->h_ctl->frame;
    });
}

slab_status slab_advance_steps(slab_ctx* c, int64_t nsteps, int64_t* steps_out) {
    if (!c) return SLAB_E_ARG;
    return guard(c, [&] {
        need(nsteps >= 0, SLAB_E_ARG, "nsteps must be >= 0");
        advance(c, nsteps, false, steps_out);
    });
}

slab_status slab_advance_steps_async(slab_ctx* c, int64_t nsteps) {
    if (!c) return SLAB_E_ARG;
    return guard(c, [&] {
        need(c->uploaded, SLAB_E_STATE, "no particles uploaded");
        need(c->initial_done, SLAB_E_STATE, "call slab_initial_pass before advancing");
        need(nsteps >= 0, SLAB_E_ARG, "nsteps must be >= 0");
        enqueue_nsteps(c, nsteps);
    });
}

slab_status slab_synchronize(slab_ctx* c) {
    if (!c) return SLAB_E_ARG;
    return guard(c, [&] {
        pull_ctl(c);
        raise_device_errors(c);
    });
}

slab_status slab_download_particles(slab_ctx* c, double* x, double* v, double* vz, double* h, double* A, double* m, double* z) {
    if (!c) return SLAB_E_ARG;
    return guard(c, [&] {
        need(c->uploaded, SLAB_E_STATE, "no particles uploaded");
        c->path->download_particles(x, v, vz, h, A, m, z);
    });
}

slab_status slab_download_grid(slab_ctx* c, slab_grid_view* view) {
    if (!c || !view) return SLAB_E_ARG;
    return guard(c, [&] {
        need(c->uploaded, SLAB_E_STATE, "no particles uploaded");
        c->path->download_grid(view);
    });
}

slab_status slab_download_max(slab_ctx* c, double* h_max, double* v_max2) {
    if (!c) return SLAB_E_ARG;
    return guard(c, [&] {
        need(c->uploaded, SLAB_E_STATE, "no particles uploaded");
        c->path->download_max(h_max, v_max2);
    });
}

slab_status slab_conservation(slab_ctx* c, double out[4]) {
    if (!c || !out) return SLAB_E_ARG;
    return guard(c, [&] {
        need(c->uploaded, SLAB_E_STATE, "no particles uploaded");
        c->path->conservation(out);
    });
}

slab_status slab_frame_capture(slab_ctx* c, int32_t slot) {
    if (!c) return SLAB_E_ARG;
    return guard(c, [&] {
        need(slot == 0 || slot == 1, SLAB_E_ARG, "frame slot must be 0 or 1");
        need(c->uploaded, SLAB_E_STATE, "no particles uploaded");
        need(c->initial_done, SLAB_E_STATE, "call slab_initial_pass before capturing a frame");
        pull_ctl(c);
        raise_device_errors(c);
        FrameSlot& F = c->frames[slot];
        if (F.pending) {  // this slot's previous copy must be over before its buffers are reused
            SLAB_CUDA(cudaEventSynchronize(F.copied));
            F.pending = false;
        }
        const int32_t* box = c->h_ctl->box;
        const int64_t nI = (int64_t)box[1] - box[0] + 1, nJ = (int64_t)box[3] - box[2] + 1;
        const int64_t nodes = nI > 0 && nJ > 0 ? nI * nJ : 0;
        const size_t need_f = (size_t)c->Np * 8 + (size_t)nodes * 6;
        if (need_f > F.cap) {
            if (F.host) cudaFreeHost(F.host);
            F.host = nullptr;
            F.cap = 0;
            F.dev = dalloc<float>(need_f);
            void* h = nullptr;
            SLAB_CUDA(cudaMallocHost(&h, need_f * sizeof(float)));
            F.host = static_cast<float*>(h);
            F.cap = need_f;
        }
        if (!F.packed) {
            SLAB_CUDA(cudaEventCreateWithFlags(&F.packed, cudaEventDisableTiming));
            SLAB_CUDA(cudaEventCreateWithFlags(&F.copied, cudaEventDisableTiming));
        }
        if (!c->copy_stream) SLAB_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
        c->path->pack_frame(F.dev.get(), F.dev.get() + (size_t)c->Np * 8, box);
        // the copy runs on its own stream, beside the steps enqueued after this call
        SLAB_CUDA(cudaEventRecord(F.packed, c->stream));
        SLAB_CUDA(cudaStreamWaitEvent(c->copy_stream, F.packed, 0));
        SLAB_CUDA(cudaMemcpyAsync(F.host, F.dev.get(), need_f * sizeof(float), cudaMemcpyDeviceToHost, c->copy_stream));
        SLAB_CUDA(cudaEventRecord(F.copied, c->copy_stream));
        F.pending = true;
        slab_frame& m = F.meta;
        m.frame = c->h_ctl->frame;
        m.Np = c->Np;
        m.time = c->h_ctl->time;
        m.particles = F.host;
        m.Nx = (int32_t)nI;
        m.Ny = (int32_t)nJ;
        m.i_off = box[0];
        m.j_off = box[2];
        m.grid = F.host + (size_t)c->Np * 8;
    });
}

slab_status slab_frame_wait(slab_ctx* c, int32_t slot, slab_frame* out) {
    // touches only the slot, so a writer thread may call it while another
    // thread advances the context; its error message goes to this thread's
    // slab_last_error(NULL)
    if (!c || !out || (slot != 0 && slot != 1)) {
        set_thread_error("slab_frame_wait: null argument or slot not 0/1");
        return SLAB_E_ARG;
    }
    FrameSlot& F = c->frames[slot];
    if (!F.pending && !F.host) {
        set_thread_error("slab_frame_wait: nothing captured in this slot");
        return SLAB_E_STATE;
    }
    if (F.pending) {
        const cudaError_t e = cudaEventSynchronize(F.copied);
        if (e != cudaSuccess) {
            set_thread_error(std::string("slab_frame_wait: ") + cudaGetErrorString(e));
            return SLAB_E_CUDA;
        }
    }
    *out = F.meta;
    return SLAB_OK;
}

slab_status slab_moments(slab_ctx* c, double out[6]) {
    if (!c || !out) return SLAB_E_ARG;
    return guard(c, [&] {
        need(c->uploaded, SLAB_E_STATE, "no particles uploaded");
        c->path->moments(out);
    });
}

slab_status slab_get_state(slab_ctx* c, double* time, double* dt, int32_t* frame, int64_t* steps) {
    if (!c) return SLAB_E_ARG;
    return guard(c, [&] {
        need(c->uploaded, SLAB_E_STATE, "no particles uploaded");
        pull_ctl(c);
        if (time) *time = c->h_ctl->time;
        if (dt) *dt = c->h_ctl->dt;
        if (frame) *frame = c->h_ctl->frame;
        if (steps) *steps = c->h_ctl->steps;
    });
}

slab_status slab_set_profiling(slab_ctx* c, int32_t on) {
    if (!c) return SLAB_E_ARG;
    return guard(c, [&] {
        need(c->uploaded, SLAB_E_STATE, "no particles uploaded");
        c->path->set_profiling(on != 0);
    });
}

slab_status slab_get_phase_times(slab_ctx* c, double out[5]) {
    if (!c || !out) return SLAB_E_ARG;
    return guard(c, [&] {
        need(c->uploaded, SLAB_E_STATE, "no particles uploaded");
        c->path->phase_times(out);
    });
}

slab_status slab_work_counters(slab_ctx* c, int64_t out[2]) {
    if (!c || !out) return SLAB_E_ARG;
    return guard(c, [&] {
        need(c->uploaded, SLAB_E_STATE, "no particles uploaded");
        pull_ctl(c);
        out[0] = c->h_ctl->steps * (int64_t)c->Np;
        out[1] = (int64_t)c->h_ctl->node_steps;
    });
}

slab_status slab_launch_shapes(slab_ctx* c, int32_t out[6]) {
    if (!c || !out) return SLAB_E_ARG;
    return guard(c, [&] {
        need(c->uploaded, SLAB_E_STATE, "no particles uploaded");
        c->path->launch_shapes(out);
    });
}

slab_status slab_set_persistent(slab_ctx* c, int32_t on, int64_t limit_cycles) {
    if (!c) return SLAB_E_ARG;
    return guard(c, [&] {
        need(limit_cycles >= 0, SLAB_E_ARG, "limit_cycles must be >= 0");
        need(c->have_params && c->params.precision != SLAB_FP64_PLAIN, SLAB_E_ARG, "persistent steps need FP32_SPLIT parameters");
        if (c->path) c->path->set_persistent(on != 0, limit_cycles);
        c->persist = on != 0 ? 1 : 0;
        if (limit_cycles > 0) c->persist_limit = limit_cycles;
    });
}

int64_t slab_kernel_launches(const slab_ctx* c) {
    if (!c) return 0;
    return c->extra_launches + (c->path ? c->path->launches() : 0);
}

const char* slab_last_error(const slab_ctx* c) { return c ? c->err.c_str() : slab::t_last_error.c_str(); }

void slab_destroy(slab_ctx* c) {
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->copy_stream) {
        cudaStreamSynchronize(c->copy_stream);
        cudaStreamDestroy(c->copy_stream);
    }
    for (FrameSlot& F : c->frames) {
        if (F.host) cudaFreeHost(F.host);
        if (F.packed) cudaEventDestroy(F.packed);
        if (F.copied) cudaEventDestroy(F.copied);
        F.dev.reset();
    }
    c->path.reset();
    c->terrain.z.reset();
    c->terrain.grad.reset();
    c->terrain.cos_t.reset();
    c->terrain.dem32.reset();
    if (c->d_ctl) cudaFree(c->d_ctl);
    if (c->h_ctl) cudaFreeHost(c->h_ctl);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
}

}  // extern "C"
