// Command-line driver for the reference oracle binary (oracle/_ref/slab_ref).
//
// TEST INFRASTRUCTURE ONLY. It calls the reference's public Simulation API in
// the same order as the reference CLI (main.cpp:40-51: loadFromJSON ->
// initialize -> initializeTerrain -> initializeParticles -> simulate) and adds
// three switches the tests and the CPU baseline need:
//
//   slab_ref <config.json>                      as the reference CLI
//   slab_ref <config.json> --init-only          stop after initializeParticles
//                                                and dump frame 0 particles
//   slab_ref <config.json> --particles f.bin    replace initializeParticles by
//                                                setParticles()/setNp() with the
//                                                particle block in f.bin (same
//                                                layout as particles_frame_*.bin)
//   slab_ref <config.json> --steps N            phase driver: t=0 pass + N steps
//                                                dumped to <sim_dir>/steps.bin
//   slab_ref <config.json> --dem-bin f.bin      replace the terrain after
//                                                initializeTerrain by the DEM in
//                                                f.bin (i64 Nx, i64 Ny, f64 dx,
//                                                then Nx*Ny z doubles, i*Ny+j)
//                                                through the public setTerrain /
//                                                setDx / terrainGradients /
//                                                terrainTheta (for large DEMs
//                                                where ASCII parsing dominates)
// With SLAB_REF_NO_DUMP=1 the output hooks write nothing, so timed runs
// contain no file output.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>

#include "simulation.hpp"

using Sim = Simulation<double, Eigen::Matrix<double, 2, 1>>;

static Grid load_dem(const char* path, double& dx) {
    FILE* f = std::fopen(path, "rb");
    if (!f) throw std::runtime_error(std::string("cannot open ") + path);
    int64_t n[2];
    if (std::fread(n, sizeof n, 1, f) != 1 || std::fread(&dx, sizeof dx, 1, f) != 1) throw std::runtime_error("short DEM file");
    Grid g(static_cast<int>(n[0]), static_cast<int>(n[1]));
    for (int i = 0; i < g.Nx; ++i) g.x[i] = i * dx;
    for (int j = 0; j < g.Ny; ++j) g.y[j] = j * dx;
    const size_t cnt = static_cast<size_t>(n[0]) * static_cast<size_t>(n[1]);
    if (std::fread(g.z.data(), sizeof(double), cnt, f) != cnt) throw std::runtime_error("short DEM file");
    std::fclose(f);
    g.xllcorner = 0.;
    g.yllcorner = 0.;
    return g;
}

static Particles load_particles(const char* path, int& Np_out) {
    FILE* f = std::fopen(path, "rb");
    if (!f) throw std::runtime_error(std::string("cannot open ") + path);
    int64_t hdr[2];
    double td[2];
    if (std::fread(hdr, sizeof hdr, 1, f) != 1 || std::fread(td, sizeof td, 1, f) != 1) throw std::runtime_error("short particle file");
    const int Np = static_cast<int>(hdr[0]);
    Particles p(Np);
    auto rd2 = [&](std::vector<TV2>& a) {
        for (int k = 0; k < Np; ++k) {
            double xy[2];
            if (std::fread(xy, sizeof xy, 1, f) != 1) throw std::runtime_error("short particle file");
            a[k] = TV2(xy[0], xy[1]);
        }
    };
    auto rd = [&](std::vector<double>& a) {
        if (Np > 0 && std::fread(a.data(), sizeof(double), Np, f) != static_cast<size_t>(Np)) throw std::runtime_error("short particle file");
    };
    rd2(p.x);
    rd(p.z);
    rd2(p.v);
    rd(p.vz);
    rd(p.h);
    rd(p.A);
    rd(p.mass);
    rd(p.theta);
    for (int k = 0; k < Np; ++k) p.order[k] = k;
    std::fclose(f);
    Np_out = Np;
    return p;
}

int main(int argc, char** argv) {
    if (argc < 2) {
        std::cerr << "Usage: " << argv[0] << " <json_file> [--init-only | --particles f.bin | --steps N]" << std::endl;
        return 1;
    }
    const char* particles_file = nullptr;
    const char* dem_file = nullptr;
    bool init_only = false;
    int steps = -1;
    for (int a = 2; a < argc; ++a) {
        if (!std::strcmp(argv[a], "--init-only"))
            init_only = true;
        else if (!std::strcmp(argv[a], "--particles") && a + 1 < argc)
            particles_file = argv[++a];
        else if (!std::strcmp(argv[a], "--dem-bin") && a + 1 < argc)
            dem_file = argv[++a];
        else if (!std::strcmp(argv[a], "--steps") && a + 1 < argc)
            steps = std::atoi(argv[++a]);
        else {
            std::cerr << "unknown argument " << argv[a] << std::endl;
            return 1;
        }
    }
    Sim sim;
    try {
        sim.loadFromJSON(argv[1]);
        sim.initialize();
        sim.initializeTerrain();
        if (dem_file) {
            double dx = 0;
            Grid g = load_dem(dem_file, dx);
            sim.setDx(dx);
            sim.setTerrain(g);
            sim.terrainGradients();
            sim.terrainTheta();
        }
        if (particles_file) {
            int Np = 0;
            Particles p = load_particles(particles_file, Np);
            sim.setNp(Np);
            sim.setParticles(p);
        } else {
            sim.initializeParticles();
        }
        if (init_only) {
            sim.saveParticleData();
            return 0;
        }
        if (steps >= 0) {
            std::string s = std::to_string(steps);
            setenv("SLAB_REF_STEPS", s.c_str(), 1);
            sim.saveTerrain();
            return 0;
        }
        sim.simulate();
    } catch (const std::exception& e) {
        std::cerr << "Error: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
