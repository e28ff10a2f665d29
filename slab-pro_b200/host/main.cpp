// Command-line driver with the reference's usage (src/main.cpp:29-57):
//
//     slab_b200 <json_file> [--fp64] [--no-output] [--init-only <particles.bin>]
//
// loadFromJSON -> initialize -> initializeTerrain -> initializeParticles ->
// simulate, with the step loop on the GPU. --fp64 runs the plain FP64 GPU
// arithmetic instead of the FP32 split one; --no-output skips the .ply/.tif
// files; --init-only stops after setup and writes the initial particles as
// raw FP64 arrays (header int64 Np, int64 frame, double time, double dt; then
// x, z, v, vz, h, A, mass, theta) without touching the GPU.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>

#include "simulation.hpp"

namespace {

void write_particles_bin(const std::string& path, const slab::Particles& P) {
    std::ofstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot write " + path);
    const int64_t n = P.size(), frame = 0;
    const double t = 0.0, dt = 0.0;
    auto put = [&](const void* p, size_t bytes) { f.write(reinterpret_cast<const char*>(p), (std::streamsize)bytes); };
    put(&n, 8);
    put(&frame, 8);
    put(&t, 8);
    put(&dt, 8);
    put(P.x.data(), P.x.size() * sizeof(slab::Vec2));
    put(P.z.data(), P.z.size() * 8);
    put(P.v.data(), P.v.size() * sizeof(slab::Vec2));
    put(P.vz.data(), P.vz.size() * 8);
    put(P.h.data(), P.h.size() * 8);
    put(P.A.data(), P.A.size() * 8);
    put(P.mass.data(), P.mass.size() * 8);
    put(P.theta.data(), P.theta.size() * 8);
    if (!f) throw std::runtime_error("failed writing " + path);
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::cerr << "Usage: " << argv[0] << " <json_file> [--fp64] [--no-output] [--init-only <particles.bin>]" << std::endl;
        return 1;
    }
    std::string init_only;
    bool fp64 = false, outputs = true;
    for (int a = 2; a < argc; ++a) {
        if (!std::strcmp(argv[a], "--fp64")) fp64 = true;
        else if (!std::strcmp(argv[a], "--no-output")) outputs = false;
        else if (!std::strcmp(argv[a], "--init-only") && a + 1 < argc) init_only = argv[++a];
        else {
            std::cerr << "unknown argument " << argv[a] << std::endl;
            return 1;
        }
    }
    slab::Simulation sim;
    try {
        sim.loadFromJSON(argv[1]);
        sim.initialize();
        std::printf("Initialization complete.\n");
        sim.initializeTerrain();
        std::printf("Terrain initialized.\n");
        sim.initializeParticles();
        std::printf("Particles initialized.\n");
        if (!init_only.empty()) {
            write_particles_bin(init_only, sim.getParticles());
            return 0;
        }
        sim.setPrecision(fp64 ? SLAB_FP64_PLAIN : SLAB_FP32_SPLIT);
        sim.setWriteOutputs(outputs);
        sim.simulate();
    } catch (const std::exception& e) {
        std::cerr << "Error: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
