// Output hooks for the reference oracle binary (oracle/_ref/slab_ref).
//
// TEST INFRASTRUCTURE ONLY. The reference declares saveParticleData,
// saveGridData, saveMaxData and saveTerrain as Simulation members
// (simulation.hpp:254-257) and defines them in save_function.cpp on top of
// GDAL and tinyply, neither of which exists here. This file gives those four
// members our own definitions. Because they are members, they can read the
// private FP64 state, so instead of .ply/.tif files they write raw binary
// dumps that the tests and the golden-fixture script read:
//
//   particles_frame_<n>.bin  i64 Np, i64 frame, f64 time, f64 dt,
//                            then x[2Np] (interleaved), z, v[2Np], vz, h, A,
//                            mass, theta (each Np doubles)
//   rasters_frame_<n>.bin    i64 Nx, Ny, i_off, j_off, frame, f64 time, f64 dt,
//                            then h, mass, v[2], vz, flip[2] on the remeshed grid
//   max_values.bin           i64 Nx, Ny, then h_max, v_max2 over the terrain
//
// With SLAB_REF_FRAME_TIMERS=1, saveParticleData also prints the sum of the
// reference's per-phase timers at every frame (the benchmark's reference arm).
//
// saveTerrain() is never called by the reference itself; here it is a
// phase-level driver: it runs the t=0 pass and SLAB_REF_STEPS steps of the
// reference's own private step functions and writes every step's state to
// <sim_dir>/steps.bin (see write_step below).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <iomanip>
#include <sstream>
#include <stdexcept>

#include "polygon_tools.hpp"
#include "simulation.hpp"

namespace fs = std::filesystem;

std::vector<TV2> loadPolygonFromShapefile(const std::string&) {
    throw std::runtime_error("POLYGON release needs GDAL/OGR, which the oracle build does not have");
}
bool isPointInPolygon(T, T, const std::vector<TV2>&) {
    return false;
}
T computePolygonArea(const std::vector<TV2>&) {
    return 0.0;
}

namespace {

struct Out {
    FILE* f;
    explicit Out(const fs::path& p, const char* mode = "wb") : f(std::fopen(p.string().c_str(), mode)) {
        if (!f) throw std::runtime_error("cannot open " + p.string());
    }
    ~Out() {
        if (f) std::fclose(f);
    }
    void i64(int64_t v) { std::fwrite(&v, sizeof v, 1, f); }
    void f64(double v) { std::fwrite(&v, sizeof v, 1, f); }
    void vec(const std::vector<double>& a, size_t n) { std::fwrite(a.data(), sizeof(double), n, f); }
    void vec2(const std::vector<TV2>& a, size_t n) {
        for (size_t k = 0; k < n; ++k) {
            f64(a[k](0));
            f64(a[k](1));
        }
    }
};

std::string frame_name(const char* stem, int padding, int frame, const char* ext) {
    std::ostringstream ss;
    ss << stem << std::setw(padding) << std::setfill('0') << frame << ext;
    return ss.str();
}

}  // namespace

static bool no_dump() {
    const char* e = std::getenv("SLAB_REF_NO_DUMP");
    return e && e[0] == '1';
}

// SLAB_REF_FRAME_TIMERS=1: at every output frame, print the sum of the
// reference's own per-phase timers so far. simulate() prints the frame's step
// count right after this hook, so a benchmark can time the steps between two
// frames (for instance, after untimed warm-up steps that end at frame 1).
static bool frame_timers() {
    const char* e = std::getenv("SLAB_REF_FRAME_TIMERS");
    return e && e[0] == '1';
}

template <typename T_, typename TV2_> void Simulation<T_, TV2_>::saveParticleData() const {
    if (frame_timers()) {
        std::printf("Phase seconds so far: %.9f\n",
                    (double)(runtime_updateDt + runtime_sort + runtime_remesh + runtime_P2G + runtime_computeGridVelocity + runtime_G2P));
        std::fflush(stdout);
    }
    if (no_dump()) return;
    Out o(particle_path / frame_name("particles_frame_", padding, frame, ".bin"));
    o.i64(Np);
    o.i64(frame);
    o.f64(time);
    o.f64(dt);
    o.vec2(particles.x, Np);
    o.vec(particles.z, Np);
    o.vec2(particles.v, Np);
    o.vec(particles.vz, Np);
    o.vec(particles.h, Np);
    o.vec(particles.A, Np);
    o.vec(particles.mass, Np);
    o.vec(particles.theta, Np);
}

template <typename T_, typename TV2_> void Simulation<T_, TV2_>::saveGridData() const {
    if (no_dump()) return;
    Out o(raster_path / frame_name("rasters_frame_", padding, frame, ".bin"));
    const size_t n = static_cast<size_t>(grid.Nx) * grid.Ny;
    o.i64(grid.Nx);
    o.i64(grid.Ny);
    o.i64(grid_i_offset);
    o.i64(grid_j_offset);
    o.i64(frame);
    o.f64(time);
    o.f64(dt);
    o.vec(grid.h, n);
    o.vec(grid.mass, n);
    o.vec2(grid.v, n);
    o.vec(grid.vz, n);
    o.vec2(grid.flip, n);
}

template <typename T_, typename TV2_> void Simulation<T_, TV2_>::saveMaxData() const {
    if (no_dump()) return;
    Out o(sim_dir_path / "max_values.bin");
    const size_t n = static_cast<size_t>(terrain.Nx) * terrain.Ny;
    o.i64(terrain.Nx);
    o.i64(terrain.Ny);
    o.vec(terrain.h_max, n);
    o.vec(terrain.v_max2, n);
}

// Phase-level driver. steps.bin holds, for the t=0 pass (record 0) and for
// each following step k=1..SLAB_REF_STEPS:
//   i64 k, f64 time (after the step), f64 dt,
//   particle block as in particles_frame_*.bin (without the header),
//   grid header i64 Nx, Ny, i_off, j_off and grid block as in rasters_frame_*,
//   terrain h_max and v_max2 (terrain.Nx*terrain.Ny doubles each).
template <typename T_, typename TV2_> void Simulation<T_, TV2_>::saveTerrain() const {
    const char* env = std::getenv("SLAB_REF_STEPS");
    const int nsteps = env ? std::atoi(env) : 0;
    auto* self = const_cast<Simulation*>(this);
    Out o(sim_dir_path / "steps.bin");
    o.i64(Np);
    o.i64(terrain.Nx);
    o.i64(terrain.Ny);
    o.i64(nsteps);
    auto write_step = [&](int k) {
        o.i64(k);
        o.f64(time);
        o.f64(dt);
        o.vec2(particles.x, Np);
        o.vec(particles.z, Np);
        o.vec2(particles.v, Np);
        o.vec(particles.vz, Np);
        o.vec(particles.h, Np);
        o.vec(particles.A, Np);
        o.vec(particles.mass, Np);
        o.vec(particles.theta, Np);
        const size_t n = static_cast<size_t>(grid.Nx) * grid.Ny;
        o.i64(grid.Nx);
        o.i64(grid.Ny);
        o.i64(grid_i_offset);
        o.i64(grid_j_offset);
        o.vec(grid.h, n);
        o.vec(grid.mass, n);
        o.vec2(grid.v, n);
        o.vec(grid.vz, n);
        o.vec2(grid.flip, n);
        const size_t nt = static_cast<size_t>(terrain.Nx) * terrain.Ny;
        o.vec(terrain.h_max, nt);
        o.vec(terrain.v_max2, nt);
    };
    // t = 0 pass, as in simulate() (simulation.cpp:493-495)
    self->remesh();
    self->P2G();
    self->computeGridVelocity();
    write_step(0);
    for (int k = 1; k <= nsteps; ++k) {
        self->advanceStep(k);
        self->time += self->dt;
        if (self->output_dt * (self->frame + 1) - self->time < 1e-13) self->frame++;
        write_step(k);
    }
}

template class Simulation<double, Eigen::Matrix<double, 2, 1>>;
