// Host-side Simulation class: the reference's public API
// (src/simulation.hpp:27-354 -- loadFromJSON, the setters and getters,
// initialize / initializeTerrain / initializeParticles / simulate, the save
// functions, readASC) over the data layouts of src/data_arrays.hpp, with the
// step loop of simulate() running on the GPU through the C ABI of
// libslab_gpu.so. Setup (terrain, release, sampling) is done on the host as
// the reference does it, so the particles handed to the device are the
// reference's own, bit for bit. Errors are std::runtime_error, as in the
// reference (caught in main, src/main.cpp:52-55).
#pragma once

#include <filesystem>
#include <functional>
#include <string>
#include <vector>

#include "data_arrays.hpp"
#include "slab_gpu.h"

namespace slab {

class Simulation {
  public:
    Simulation();
    ~Simulation();
    Simulation(const Simulation&) = delete;
    Simulation& operator=(const Simulation&) = delete;

    void loadFromJSON(const std::filesystem::path& json_path);

    // setters for simulation configuration (src/simulation.hpp:79-214)
    void setSimName(const std::string& name) { sim_name = name; }
    void setProjectDir(const std::filesystem::path& path) { project_dir_path = path; }
    void setParticlePath(const std::filesystem::path& path) { particle_path = path; }
    void setRasterPath(const std::filesystem::path& path) { raster_path = path; }
    void setDemFilePath(const std::filesystem::path& path) { dem_filepath = path; }
    void setPolygonPath(const std::filesystem::path& path) { poly.filepath = path; }
    void setNFiles(int n) { nFiles = n; }
    void setPadding(int p) { padding = p; }
    void setRho(T r) { rho = r; }
    void setH0(T h) { h0 = h; }
    void setGravity(T g) { gravity = g; }
    void setTotalTime(T t) { total_time = t; }
    void setCFL(T cfl) { C_cfl = cfl; }
    void setDt(T delta_t) { dt = delta_t; }
    void setDtMax(T dtm) { dt_max = dtm; }
    void setFlipRatio(T fr) { flip_ratio = fr; }
    void setOutputDt(T odt) { output_dt = odt; }
    void setFrame(int f) { frame = f; }
    void setFrictionType(const FrictionType& f) { friction.type = f; }
    void setFrictionCoulombMu(double mu) { friction.coulomb.mu = mu; }
    void setFrictionVoellmyMu(double mu) { friction.voellmy.mu = mu; }
    void setFrictionVoellmyXi(double xi) { friction.voellmy.xi = xi; }
    void setFrictionMuIMu1(double v) { friction.muI.mu_1 = v; }
    void setFrictionMuIMu2(double v) { friction.muI.mu_2 = v; }
    void setFrictionMuII0(double v) { friction.muI.I0 = v; }
    void setFrictionMuID(double v) { friction.muI.d = v; }
    void setFrictionMuIPhi(double v) { friction.muI.phi = v; }
    void setTerrainType(TerrainType tt) { terrain_type = tt; }
    void setTerrainLx(T l) { terrain_Lx = l; }
    void setTerrainLy(T l) { terrain_Ly = l; }
    void setDx(T delta_x) {
        dx = delta_x;
        one_over_dx = T(1) / dx;
    }
    void setOneOverDx(T oodx) {
        one_over_dx = oodx;
        dx = T(1) / one_over_dx;
    }
    void setAltZFunction(const std::function<T(const T&, const T&)>& f) { alt_z = f; }
    void setReleaseShapeType(ReleaseShapeType r) { release_shape_type = r; }
    void setRectangle(const Rectangle& r) { rect = r; }
    void setEllipse(const Ellipse& e) { ell = e; }
    void setPolygon(const Polygon& p) { poly = p; }
    void setReleaseArea(T a) { release_area = a; }
    void setReleaseHeightRasterFilepath(const std::string& p) { release_height_raster_filepath = p; }
    void setSamplingMethod(SamplingMethod s) { sampling_method = s; }
    void setNp(int np) { Np = np; }
    void setParticles(const Particles& p) {
        particles = p;
        Np = p.size();
    }
    void setGrid(const Grid& g) { grid = g; }
    void setTerrain(const Grid& t) { terrain = t; }
    // GPU arithmetic of the step loop: SLAB_FP32_SPLIT (default) or SLAB_FP64_PLAIN
    void setPrecision(slab_precision p) { precision = p; }
    // write no .ply / .tif files (benchmarks)
    void setWriteOutputs(bool on) { write_outputs = on; }

    std::filesystem::path getProjectDir() const { return project_dir_path; }
    std::string getSimName() const { return sim_name; }
    std::filesystem::path getDemFilePath() const { return dem_filepath; }
    std::filesystem::path getParticlePath() const { return particle_path; }
    std::filesystem::path getRasterPath() const { return raster_path; }
    std::filesystem::path getSimDir() const { return sim_dir_path; }
    FrictionType getFrictionType() const { return friction.type; }
    const Particles& getParticles() const { return particles; }
    const Grid& getGrid() const { return grid; }
    const Grid& getTerrain() const { return terrain; }
    int getNp() const { return Np; }
    T getTime() const { return time; }
    int getFrame() const { return frame; }
    int64_t getSteps() const { return steps; }

    // lifecycle (src/simulation.cpp:58-522)
    void initialize();
    void initializeTerrain();
    void initializeParticles();
    void simulate();

    // helpers of the reference kept with their meaning
    Vec2 rotatePoint(const Vec2& p, T angle) const;
    Vec2 particleGradients(int p) const;
    T particleSlopeAngle(int p) const;
    void terrainGradients();
    void terrainTheta();
    std::vector<T> generateGrid(T length, T dx) const;
    T getReleaseHeightFromRaster(const Vec2 position) const;

    // I/O (src/save_function.cpp): binary .ply particles, 6-band GeoTIFF grid
    // rasters per frame, 2-band max_values.tif
    void saveParticleData() const;
    void saveGridData() const;
    void saveMaxData() const;
    RasterData readASC(const std::filesystem::path& path) const;

  private:
    FrictionType parseFrictionType(const std::string& s);
    TerrainType parseTerrainType(const std::string& s);
    ReleaseShapeType parseReleaseShapeType(const std::string& s);
    void pull_frame();

    std::string sim_name;
    std::filesystem::path json_file_path, sim_dir_path, project_dir_path, particle_path, raster_path, dem_filepath;
    int nFiles = 0, padding = 0;

    T rho, h0, gravity, time = 0.0, total_time, C_cfl, dt, dt_max, flip_ratio, output_dt;
    int frame = 0;
    Friction friction;

    TerrainType terrain_type;
    T terrain_Lx, terrain_Ly, dx, one_over_dx;
    std::function<T(const T&, const T&)> alt_z;

    ReleaseShapeType release_shape_type;
    Rectangle rect;
    Ellipse ell;
    Polygon poly;
    Raster rast;
    T release_area = 0.0;
    std::string release_height_raster_filepath;
    Grid release_height_raster;

    SamplingMethod sampling_method;
    const int ppc = 4;

    int Np = 0;
    Particles particles;
    Grid grid;
    Grid terrain;

    slab_precision precision = SLAB_FP32_SPLIT;
    bool write_outputs = true;
    int64_t steps = 0;
    slab_ctx* ctx = nullptr;
};

}  // namespace slab
