// Host-side Simulation: setup as the reference does it (bit for bit), the
// step loop on the GPU through libslab_gpu.so, outputs through the writers
// of this directory. Built with -ffp-contract=off so that every FP64
// expression of the setup rounds as the reference's does.
#include "simulation.hpp"

#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <exception>
#include <mutex>
#include <thread>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <sstream>
#include <stdexcept>

#include "json.hpp"
#include "writers.hpp"

namespace fs = std::filesystem;

namespace slab {

namespace {

// quadratic B-spline N(u) (src/tools.hpp:119-128)
inline T N(T u) {
    const T a = std::abs(u);
    if (a < 0.5) return 0.75 - a * a;
    if (a < 1.5) return 0.5 * (1.5 - a) * (1.5 - a);
    return 0.0;
}

inline T wip(T xp, T yp, T xi, T yi, T ooh) { return N((xp - xi) * ooh) * N((yp - yi) * ooh); }

void check(slab_status s, const slab_ctx* c, const char* what) {
    if (s != SLAB_OK) throw std::runtime_error(std::string(what) + ": " + slab_last_error(c));
}

std::string read_file(const fs::path& p) {
    std::ifstream f(p, std::ios::binary);
    if (!f) throw std::runtime_error("JSON file not found: " + p.string());
    std::ostringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

std::string frame_name(const char* stem, int padding, int frame, const char* ext) {
    std::ostringstream ss;
    ss << stem << std::setw(padding) << std::setfill('0') << frame << ext;
    return ss.str();
}

}  // namespace

// defaults of the reference constructor (src/simulation.hpp:29-71)
Simulation::Simulation()
    : sim_name("default_sim"),
      rho(2500.0),
      h0(30.0),
      gravity(9.8045),
      total_time(80.0),
      C_cfl(0.5),
      dt(0.0),
      dt_max(0.06),
      flip_ratio(0.9),
      output_dt(5.0),
      friction{FrictionType::Coulomb, {0.531709431759}, {0.2, 200.0}, {0.2, 0.9, 0.1, 0.005, 0.6}},
      terrain_type(TerrainType::Analytical),
      terrain_Lx(5000.0),
      terrain_Ly(5000.0),
      dx(8.0),
      one_over_dx(1.0 / 8.0),
      alt_z([](const T&, const T&) { return T(0); }),
      release_shape_type(ReleaseShapeType::Rectangle),
      rect{Vec2(1200.0, 1400.0), 100.0, 80.0, 0.0},
      ell{Vec2(1200.0, 1400.0), 100.0, 80.0, 0.0},
      sampling_method(SamplingMethod::Uniform) {}

Simulation::~Simulation() {
    if (ctx) slab_destroy(ctx);
}

FrictionType Simulation::parseFrictionType(const std::string& s) {
    if (s == "COULOMB") return FrictionType::Coulomb;
    if (s == "VOELLMY") return FrictionType::Voellmy;
    if (s == "MU_I") return FrictionType::mu_I;
    throw std::runtime_error("Unknown friction type: " + s);
}

TerrainType Simulation::parseTerrainType(const std::string& s) {
    if (s == "DEM") return TerrainType::DEM;
    if (s == "ANALYTICAL") return TerrainType::Analytical;
    throw std::runtime_error("Unknown terrain type: " + s);
}

ReleaseShapeType Simulation::parseReleaseShapeType(const std::string& s) {
    if (s == "RECTANGLE") return ReleaseShapeType::Rectangle;
    if (s == "ELLIPSE") return ReleaseShapeType::Ellipse;
    if (s == "POLYGON") return ReleaseShapeType::Polygon;
    if (s == "RASTER") return ReleaseShapeType::Raster;
    throw std::runtime_error("Unknown release shape type: " + s);
}

// the input schema of src/simulation.cpp:118-208
void Simulation::loadFromJSON(const fs::path& json_path) {
    json_file_path = json_path;
    if (!fs::exists(json_path)) throw std::runtime_error("JSON file not found: " + json_path.string());
    const json::Value j = json::parse(read_file(json_path));

    project_dir_path = j.at("project_dir").get_string();
    sim_name = j.at("sim_name").get_string();

    const auto& phys = j.at("physical_params");
    gravity = phys.at("gravity").get_double();
    rho = phys.at("rho").get_double();

    const auto& tp = j.at("time_params");
    output_dt = tp.at("output_dt").get_double();
    total_time = tp.at("total_time").get_double();

    const auto& np = j.at("numerical_params");
    C_cfl = np.at("C_cfl").get_double();
    dt_max = np.at("dt_max").get_double();
    flip_ratio = np.at("flip_ratio").get_double();
    const std::string method = np.at("sampling_method").get_string();
    if (method == "UNIFORM") sampling_method = SamplingMethod::Uniform;
    else if (method == "POISSON") sampling_method = SamplingMethod::Poisson;
    else throw std::runtime_error("Unknown sampling method: " + method);

    const auto& fr = j.at("friction");
    friction.type = parseFrictionType(fr.at("type").get_string());
    if (friction.type == FrictionType::Coulomb) {
        friction.coulomb.mu = fr.at("coulomb").at("mu").get_double();
    } else if (friction.type == FrictionType::Voellmy) {
        friction.voellmy.mu = fr.at("voellmy").at("mu").get_double();
        friction.voellmy.xi = fr.at("voellmy").at("xi").get_double();
    } else {
        const auto& m = fr.at("mu_I");
        friction.muI.mu_1 = m.at("mu_1").get_double();
        friction.muI.mu_2 = m.at("mu_2").get_double();
        friction.muI.I0 = m.at("I0").get_double();
        friction.muI.d = m.at("d").get_double();
        friction.muI.phi = m.at("phi").get_double();
    }

    const auto& tr = j.at("terrain");
    terrain_type = parseTerrainType(tr.at("type").get_string());
    if (terrain_type == TerrainType::DEM) {
        dem_filepath = tr.at("dem").at("filepath").get_string();
    } else {
        terrain_Lx = tr.at("analytical").at("Lx").get_double();
        terrain_Ly = tr.at("analytical").at("Ly").get_double();
        dx = tr.at("analytical").at("dx").get_double();
        // the reference's hard-coded analytical terrain: a 5-degree plane falling in +x and +y
        alt_z = [](const T& x, const T& y) -> T {
            const double th = 5.0 * M_PI / 180.0;
            return -x * std::tan(th) - y * std::tan(th);
        };
    }

    const auto& rel = j.at("release");
    release_shape_type = parseReleaseShapeType(rel.at("type").get_string());
    h0 = rel.at("h0").get_double();
    if (release_shape_type == ReleaseShapeType::Rectangle) {
        const auto& r = rel.at("rectangle");
        rect.center = Vec2(r.at("center")[0].get_double(), r.at("center")[1].get_double());
        rect.Lx = r.at("Lx").get_double();
        rect.Ly = r.at("Ly").get_double();
        rect.rotation = r.at("rotation_deg").get_double() * M_PI / 180.0;
    } else if (release_shape_type == ReleaseShapeType::Ellipse) {
        const auto& e = rel.at("ellipse");
        ell.center = Vec2(e.at("center")[0].get_double(), e.at("center")[1].get_double());
        ell.rx = e.at("rx").get_double();
        ell.ry = e.at("ry").get_double();
        ell.rotation = e.at("rotation_deg").get_double() * M_PI / 180.0;
    } else if (release_shape_type == ReleaseShapeType::Polygon) {
        poly.filepath = rel.at("polygon").at("filepath").get_string();
    } else {
        rast.filepath = rel.at("raster").at("filepath").get_string();
        rast.h_min = rel.at("raster").at("h_min").get_double();
    }
}

// src/simulation.cpp:58-88 and createSimulationDirectories (src/tools.cpp:28-52)
void Simulation::initialize() {
    sim_dir_path = project_dir_path / sim_name;
    try {
        if (fs::create_directories(sim_dir_path)) std::cout << "Directory " << sim_dir_path << " has been created." << std::endl;
        else std::cerr << "Directory " << sim_dir_path << " already exists or could not be created." << std::endl;
        fs::create_directories(sim_dir_path / "rasters");
        fs::create_directories(sim_dir_path / "particles");
    } catch (const std::exception& e) {
        std::cerr << "Filesystem error: " << e.what() << std::endl;
    }
    particle_path = sim_dir_path / "particles";
    raster_path = sim_dir_path / "rasters";
    nFiles = static_cast<int>(std::ceil(total_time / output_dt));
    padding = static_cast<int>(std::floor(std::log10(nFiles))) + 1;
    if (!json_file_path.empty()) {
        try {
            fs::copy_file(json_file_path, sim_dir_path / json_file_path.filename(), fs::copy_options::overwrite_existing);
        } catch (const std::exception& e) {
            std::cerr << "Failed to copy JSON file: " << e.what() << "\n";
        }
    }
    time = 0.0;
    frame = 0;
    steps = 0;
}

// src/complex_terrain.cpp:31-65: the ESRI ASCII grid, rows stored from the
// south edge (z[i * nrows + j], j = 0 the last row of the file); nodata is
// not masked
namespace {

// Binary cache of a parsed .asc file, written next to it as <file>.slabbin:
// the header values, the source file's size and modification time, and the
// heights in the terrain's i * nrows + j order. A later read of the same,
// unchanged file loads the doubles the parse produced instead of parsing the
// text again (the ASCII parse of a 28 MB DEM takes seconds).
constexpr char CACHE_MAGIC[8] = {'S', 'L', 'A', 'B', 'D', 'E', 'M', '1'};
struct CacheHeader {
    char magic[8];
    int64_t src_size, src_mtime;
    int32_t ncols, nrows;
    double xllcorner, yllcorner, cellsize, nodata;
};

int64_t mtime_of(const fs::path& p) {
    std::error_code ec;
    const auto t = fs::last_write_time(p, ec);
    return ec ? -1 : (int64_t)t.time_since_epoch().count();
}

bool read_asc_cache(const fs::path& src, RasterData& r) {
    std::error_code ec;
    const fs::path cp = fs::path(src.string() + ".slabbin");
    if (!fs::exists(cp, ec)) return false;
    std::ifstream f(cp, std::ios::binary);
    CacheHeader h{};
    if (!f.read(reinterpret_cast<char*>(&h), sizeof h)) return false;
    if (std::memcmp(h.magic, CACHE_MAGIC, 8) != 0 || h.ncols <= 0 || h.nrows <= 0) return false;
    if (h.src_size != (int64_t)fs::file_size(src, ec) || ec || h.src_mtime != mtime_of(src)) return false;
    r.ncols = h.ncols;
    r.nrows = h.nrows;
    r.xllcorner = h.xllcorner;
    r.yllcorner = h.yllcorner;
    r.cellsize = h.cellsize;
    r.nodata = h.nodata;
    r.z.resize((size_t)r.ncols * r.nrows);
    if (!f.read(reinterpret_cast<char*>(r.z.data()), (std::streamsize)(r.z.size() * sizeof(double)))) return false;
    return true;
}

void write_asc_cache(const fs::path& src, const RasterData& r) {
    std::error_code ec;
    CacheHeader h{};
    std::memcpy(h.magic, CACHE_MAGIC, 8);
    h.src_size = (int64_t)fs::file_size(src, ec);
    if (ec) return;
    h.src_mtime = mtime_of(src);
    h.ncols = r.ncols;
    h.nrows = r.nrows;
    h.xllcorner = r.xllcorner;
    h.yllcorner = r.yllcorner;
    h.cellsize = r.cellsize;
    h.nodata = r.nodata;
    const fs::path cp = fs::path(src.string() + ".slabbin"), tmp = fs::path(cp.string() + ".tmp");
    {
        std::ofstream f(tmp, std::ios::binary);
        if (!f) return;  // read-only directory: no cache, nothing else changes
        f.write(reinterpret_cast<const char*>(&h), sizeof h);
        f.write(reinterpret_cast<const char*>(r.z.data()), (std::streamsize)(r.z.size() * sizeof(double)));
        if (!f) {
            f.close();
            fs::remove(tmp, ec);
            return;
        }
    }
    fs::rename(tmp, cp, ec);
    if (ec) fs::remove(tmp, ec);
}

}  // namespace

// src/complex_terrain.cpp:31-65: header, then the rows from the north edge
// down, stored so that j grows northwards. The values are parsed with
// strtod, as the stream extraction of the reference does, so the doubles are
// the same; the parsed raster is cached in binary next to the file.
RasterData Simulation::readASC(const fs::path& path) const {
    RasterData r;
    if (read_asc_cache(path, r)) {
        for (int i = 0; i < r.ncols; ++i) r.x.push_back(i * r.cellsize);
        for (int j = 0; j < r.nrows; ++j) r.y.push_back(j * r.cellsize);
        return r;
    }
    std::ifstream file(path, std::ios::binary);
    if (!file.is_open()) throw std::runtime_error("Failed to open ASC file: " + path.string());
    std::string text((std::istreambuf_iterator<char>(file)), std::istreambuf_iterator<char>());
    std::istringstream head(text);
    std::string key;
    head >> key >> r.ncols >> key >> r.nrows >> key >> r.xllcorner >> key >> r.yllcorner >> key >> r.cellsize >> key >> r.nodata;
    if (!head || r.ncols <= 0 || r.nrows <= 0) throw std::runtime_error("Bad ASC header: " + path.string());
    const std::streamoff off = head.tellg();
    for (int i = 0; i < r.ncols; ++i) r.x.push_back(i * r.cellsize);
    for (int j = 0; j < r.nrows; ++j) r.y.push_back(j * r.cellsize);
    r.z.resize((size_t)r.ncols * r.nrows);
    const char* p = text.c_str() + (off < 0 ? text.size() : (size_t)off);
    for (int j = r.nrows - 1; j >= 0; --j)
        for (int i = 0; i < r.ncols; ++i) {
            char* end = nullptr;
            const double v = std::strtod(p, &end);
            if (end == p) throw std::runtime_error("ASC file ended early: " + path.string());
            r.z[ind(i, j, r.nrows)] = v;
            p = end;
        }
    write_asc_cache(path, r);
    return r;
}

std::vector<T> Simulation::generateGrid(T length, T step) const {
    std::vector<T> g;
    int idx = 0;
    T x = 0.0;
    g.push_back(x);
    while (x < length) {
        ++idx;
        x = static_cast<T>(idx) * step;
        g.push_back(x);
    }
    return g;
}

// src/simulation.cpp:210-257
void Simulation::initializeTerrain() {
    if (terrain_type == TerrainType::DEM) {
        RasterData r = readASC(dem_filepath);
        terrain = Grid(r.ncols, r.nrows);
        terrain.x = r.x;
        terrain.y = r.y;
        terrain.z = r.z;
        terrain.xllcorner = r.xllcorner;
        terrain.yllcorner = r.yllcorner;
        terrain.nodata = r.nodata;
        dx = r.cellsize;
        one_over_dx = 1. / dx;
    } else {
        one_over_dx = 1. / dx;
        const auto tx = generateGrid(terrain_Lx, dx), ty = generateGrid(terrain_Ly, dx);
        terrain = Grid((int)tx.size(), (int)ty.size());
        terrain.x = tx;
        terrain.y = ty;
        for (int i = 0; i < terrain.Nx; ++i)
            for (int j = 0; j < terrain.Ny; ++j) terrain.z[ind(i, j, terrain.Ny)] = alt_z(terrain.x[i], terrain.y[j]);
    }
    terrainGradients();
    terrainTheta();
    std::fill(terrain.h_max.begin(), terrain.h_max.end(), 0.);
    std::fill(terrain.v_max2.begin(), terrain.v_max2.end(), 0.);
}

// src/complex_terrain.cpp:84-100: the cell gradient, stored at the cell's
// lower-left node; the last row and column stay zero
void Simulation::terrainGradients() {
    const int Ny = terrain.Ny;
    const T* z = terrain.z.data();
    for (int i = 0; i < terrain.Nx - 1; ++i)
        for (int j = 0; j < Ny - 1; ++j) {
            const T dzx = (z[ind(i + 1, j, Ny)] + z[ind(i + 1, j + 1, Ny)] - z[ind(i, j, Ny)] - z[ind(i, j + 1, Ny)]) / 2. * one_over_dx;
            const T dzy = (z[ind(i, j + 1, Ny)] + z[ind(i + 1, j + 1, Ny)] - z[ind(i, j, Ny)] - z[ind(i + 1, j, Ny)]) / 2. * one_over_dx;
            terrain.gradients[ind(i, j, Ny)] = Vec2(dzx, dzy);
        }
}

// src/complex_terrain.cpp:102-111
void Simulation::terrainTheta() {
    for (size_t k = 0; k < terrain.theta.size(); ++k) terrain.theta[k] = std::atan(std::sqrt(terrain.gradients[k].squaredNorm()));
}

// src/complex_terrain.cpp:113-130 (slope of the cell holding the particle)
T Simulation::particleSlopeAngle(int p) const {
    const Vec2& x = particles.x[p];
    const int i = static_cast<int>(std::floor((x(0) - terrain.x[0]) * one_over_dx));
    const int j = static_cast<int>(std::floor((x(1) - terrain.y[0]) * one_over_dx));
    return terrain.theta[ind(i, j, terrain.Ny)];
}

Vec2 Simulation::particleGradients(int p) const {
    const Vec2& x = particles.x[p];
    const int i = static_cast<int>(std::floor((x(0) - terrain.x[0]) * one_over_dx));
    const int j = static_cast<int>(std::floor((x(1) - terrain.y[0]) * one_over_dx));
    return terrain.gradients[ind(i, j, terrain.Ny)];
}

Vec2 Simulation::rotatePoint(const Vec2& p, T angle) const {
    const T c = std::cos(angle), s = std::sin(angle);
    return Vec2(c * p(0) - s * p(1), s * p(0) + c * p(1));
}

// src/complex_terrain.cpp:132-183: bilinear release height, 0 outside the
// raster, next to nodata, or where it is not positive. The bound test uses
// the raster's last coordinate as stored (relative to the terrain origin),
// as the reference does.
T Simulation::getReleaseHeightFromRaster(const Vec2 position) const {
    const Grid& R = release_height_raster;
    if (R.Nx == 0 || R.Ny == 0) return 0.0;
    const T xr = position(0) - R.x[0], yr = position(1) - R.y[0];
    if (xr < 0 || yr < 0 || xr >= R.x.back() || yr >= R.y.back()) return 0.0;
    const T dxl = R.x[1] - R.x[0], dyl = R.y[1] - R.y[0];
    const int i = static_cast<int>(std::floor(xr / dxl)), j = static_cast<int>(std::floor(yr / dyl));
    if (i < 0 || j < 0 || i >= R.Nx - 1 || j >= R.Ny - 1) return 0.0;
    const T fx = (xr - i * dxl) / dxl, fy = (yr - j * dyl) / dyl;
    const T z00 = R.z[ind(i, j, R.Ny)], z10 = R.z[ind(i + 1, j, R.Ny)], z01 = R.z[ind(i, j + 1, R.Ny)], z11 = R.z[ind(i + 1, j + 1, R.Ny)];
    const T nd = R.nodata;
    if (std::abs(z00 - nd) < 1e-6 || std::abs(z10 - nd) < 1e-6 || std::abs(z01 - nd) < 1e-6 || std::abs(z11 - nd) < 1e-6) return 0.0;
    const T z0 = z00 * (1.0 - fx) + z10 * fx;
    const T z1 = z01 * (1.0 - fx) + z11 * fx;
    const T hgt = z0 * (1.0 - fy) + z1 * fy;
    return hgt > 0.0 ? hgt : 0.0;
}

// src/simulation.cpp:259-476
void Simulation::initializeParticles() {
    std::vector<Vec2> samples, pos;
    T x_min = 0, x_max = 0, y_min = 0, y_max = 0, volume = 0;
    switch (release_shape_type) {
        case ReleaseShapeType::Rectangle: {
            const T diag = std::sqrt(rect.Lx * rect.Lx + rect.Ly * rect.Ly) / 2.;
            x_min = rect.center(0) - diag;
            x_max = rect.center(0) + diag;
            y_min = rect.center(1) - diag;
            y_max = rect.center(1) + diag;
            release_area = rect.Lx * rect.Ly;
            break;
        }
        case ReleaseShapeType::Ellipse: {
            const T big = std::max(ell.rx, ell.ry);
            x_min = ell.center(0) - big;
            x_max = ell.center(0) + big;
            y_min = ell.center(1) - big;
            y_max = ell.center(1) + big;
            release_area = M_PI * ell.rx * ell.ry;
            break;
        }
        case ReleaseShapeType::Polygon:
            throw std::runtime_error("POLYGON releases need a shapefile reader, which this build does not have; use RASTER");
        case ReleaseShapeType::Raster: {
            const RasterData r = readASC(rast.filepath);
            Grid& R = release_height_raster;
            R = Grid(r.ncols, r.nrows);
            for (int i = 0; i < r.ncols; ++i) R.x[i] = r.xllcorner - terrain.xllcorner + i * r.cellsize;
            for (int j = 0; j < r.nrows; ++j) R.y[j] = r.yllcorner - terrain.yllcorner + j * r.cellsize;
            R.z = r.z;
            R.xllcorner = r.xllcorner;
            R.yllcorner = r.yllcorner;
            R.nodata = r.nodata;
            x_min = r.xllcorner - terrain.xllcorner;
            y_min = r.yllcorner - terrain.yllcorner;
            x_max = x_min + r.cellsize * (r.ncols - 1);
            y_max = y_min + r.cellsize * (r.nrows - 1);
            int count = 0;
            const T cell_area = r.cellsize * r.cellsize;
            for (int j = 0; j < r.nrows; ++j)
                for (int i = 0; i < r.ncols; ++i) {
                    const T hc = r.z[ind(i, j, r.nrows)];
                    if (hc >= rast.h_min && hc > 0.) {
                        ++count;
                        volume += hc * cell_area;
                    }
                }
            release_area = count * cell_area;
            break;
        }
    }
    if (release_shape_type != ReleaseShapeType::Raster) volume = release_area * h0;

    x_min = std::floor(x_min * one_over_dx) * dx;
    x_max = std::ceil(x_max * one_over_dx) * dx;
    y_min = std::floor(y_min * one_over_dx) * dx;
    y_max = std::ceil(y_max * one_over_dx) * dx;

    if (sampling_method == SamplingMethod::Uniform) {
        const int nxc = static_cast<int>(std::round((x_max - x_min) * one_over_dx));
        const int nyc = static_cast<int>(std::round((y_max - y_min) * one_over_dx));
        const T dxp[4] = {0.25, 0.75, 0.25, 0.75}, dyp[4] = {0.25, 0.25, 0.75, 0.75};
        samples.reserve((size_t)std::max(nxc, 0) * std::max(nyc, 0) * ppc);
        for (int i = 0; i < nxc; ++i)
            for (int j = 0; j < nyc; ++j)
                for (int d = 0; d < ppc; ++d) samples.push_back(Vec2(((double)i + dxp[d]) * dx, ((double)j + dyp[d]) * dx));
    } else {
        // the reference's Poisson_disk sampler (src/poisson_disk_sampling.hpp:37): radius from dx and 4 particles
        // per cell, 30 candidates, the C library's rand() seeded with 1
        const T r = std::sqrt(15.0 / 24.0 * dx * dx / ppc);
        int64_t n = 0;
        check(slab_poisson_disk(x_max - x_min, y_max - y_min, r, 30, 0, nullptr, 0, &n), nullptr, "Poisson sampling");
        std::vector<double> xy(2 * (size_t)n);
        check(slab_poisson_disk(x_max - x_min, y_max - y_min, r, 30, 0, xy.data(), n, &n), nullptr, "Poisson sampling");
        samples.resize((size_t)n);
        for (int64_t q = 0; q < n; ++q) samples[q] = Vec2(xy[2 * q], xy[2 * q + 1]);
    }

    for (const Vec2& p : samples) {
        const Vec2 s = p + Vec2(x_min, y_min);
        bool keep = false;
        switch (release_shape_type) {
            case ReleaseShapeType::Rectangle: {
                const Vec2 l = rotatePoint(s - rect.center, -rect.rotation);
                keep = std::abs(l(0)) <= rect.Lx / 2. && std::abs(l(1)) <= rect.Ly / 2.;
                break;
            }
            case ReleaseShapeType::Ellipse: {
                const Vec2 l = rotatePoint(s - ell.center, -ell.rotation);
                keep = std::pow(l(0) / ell.rx, 2.) + std::pow(l(1) / ell.ry, 2.) <= 1.;
                break;
            }
            case ReleaseShapeType::Raster: {
                const T hr = getReleaseHeightFromRaster(s);
                keep = hr >= rast.h_min && hr > 0.;
                break;
            }
            case ReleaseShapeType::Polygon: break;
        }
        if (keep) pos.push_back(s);
    }

    Np = static_cast<int>(pos.size());
    particles = Particles(Np);
    std::vector<T> h_init(Np, h0);
    T sum_h = 0.0;
    for (int p = 0; p < Np; ++p) {
        if (release_shape_type == ReleaseShapeType::Raster) h_init[p] = getReleaseHeightFromRaster(pos[p]);
        sum_h += h_init[p];
    }
    const T A_init = volume / sum_h;
    for (int p = 0; p < Np; ++p) {
        particles.x[p] = pos[p];
        particles.order[p] = p;
        particles.h[p] = h_init[p];
        particles.A[p] = A_init;
        particles.mass[p] = rho * particles.h[p] * particles.A[p];
        // the 4x4 node window of the z interpolation holds the particle's cell
        // (the slope angle's node) too: check it before either is read
        const Vec2& xp = particles.x[p];
        const int ib = static_cast<int>((xp(0) - terrain.x[0]) * one_over_dx) - 1;
        const int jb = static_cast<int>((xp(1) - terrain.y[0]) * one_over_dx) - 1;
        if (ib < 0 || jb < 0 || ib + 3 >= terrain.Nx || jb + 3 >= terrain.Ny)
            throw std::runtime_error("release reaches the terrain edge (particle " + std::to_string(p) + ")");
        particles.theta[p] = particleSlopeAngle(p);
        for (int i = ib; i < ib + 4; ++i)
            for (int j = jb; j < jb + 4; ++j) {
                const T w = wip(xp(0), xp(1), terrain.x[i], terrain.y[j], one_over_dx);
                particles.z[p] += terrain.z[ind(i, j, terrain.Ny)] * w;
            }
    }
    T total_volume = 0.0;
    for (int p = 0; p < Np; ++p) total_volume += particles.h[p] * particles.A[p];
    std::cout << "Total volume: " << total_volume << std::endl;
    std::cout << "Number of particles: " << Np << std::endl;
}

// the current frame's particles and grid from the device into the reference's containers
void Simulation::pull_frame() {
    check(slab_download_particles(ctx, &particles.x[0](0), &particles.v[0](0), particles.vz.data(), particles.h.data(), particles.A.data(),
                                  particles.mass.data(), particles.z.data()),
          ctx, "slab_download_particles");
    slab_grid_view gv{};
    check(slab_download_grid(ctx, &gv), ctx, "slab_download_grid");  // sizes only
    grid.resize(gv.Nx, gv.Ny);
    for (int i = 0; i < gv.Nx; ++i) grid.x[i] = terrain.x[gv.i_off + i];
    for (int j = 0; j < gv.Ny; ++j) grid.y[j] = terrain.y[gv.j_off + j];
    gv.cap_nodes = (int64_t)gv.Nx * gv.Ny;
    gv.h = grid.h.data();
    gv.mass = grid.mass.data();
    gv.v = gv.cap_nodes ? &grid.v[0](0) : nullptr;
    gv.vz = grid.vz.data();
    gv.flip = gv.cap_nodes ? &grid.flip[0](0) : nullptr;
    gv.F = gv.cap_nodes ? &grid.F[0](0) : nullptr;
    gv.a = gv.cap_nodes ? &grid.a[0](0) : nullptr;
    if (gv.cap_nodes > 0) check(slab_download_grid(ctx, &gv), ctx, "slab_download_grid");
}

namespace {

// Writes the frames captured by slab_frame_capture on its own thread, so that
// the files of frame k are written while the GPU runs frame k+1's steps.
// Frame k uses capture slot k % 2; the slot can be captured again once job
// k has been written (wait_written).
class FrameWriter {
  public:
    using WriteFn = std::function<void(const slab_frame&)>;
    FrameWriter(slab_ctx* ctx, WriteFn fn) : ctx_(ctx), fn_(std::move(fn)), th_([this] { run(); }) {}
    ~FrameWriter() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        if (th_.joinable()) th_.join();
    }
    // queue job k (frames are numbered 0, 1, ... in capture order)
    void push(int64_t k) {
        {
            std::lock_guard<std::mutex> lk(mu_);
            jobs_.push_back(k);
        }
        cv_.notify_all();
    }
    // block until job k is written (k < 0: nothing to wait for); rethrows a writer error
    void wait_written(int64_t k) {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return written_ >= k || err_; });
        if (err_) std::rethrow_exception(err_);
    }

  private:
    void run() {
        for (;;) {
            int64_t k;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || !jobs_.empty(); });
                if (jobs_.empty()) return;
                k = jobs_.front();
                jobs_.pop_front();
            }
            try {
                slab_frame f{};
                const slab_status st = slab_frame_wait(ctx_, (int32_t)(k % 2), &f);
                if (st != SLAB_OK) throw std::runtime_error(std::string("slab_frame_wait: ") + slab_last_error(nullptr));
                fn_(f);
            } catch (...) {
                std::lock_guard<std::mutex> lk(mu_);
                err_ = std::current_exception();
                cv_.notify_all();
                return;
            }
            {
                std::lock_guard<std::mutex> lk(mu_);
                written_ = k;
            }
            cv_.notify_all();
        }
    }
    slab_ctx* ctx_;
    WriteFn fn_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<int64_t> jobs_;
    int64_t written_ = -1;
    bool stop_ = false;
    std::exception_ptr err_;
    std::thread th_;  // last: starts after the members it reads
};

}  // namespace

// src/simulation.cpp:484-522 with the step loop on the GPU. Output frames are
// packed on the device and written by a writer thread while the next frame's
// steps run (slab_frame_capture / slab_frame_wait).
void Simulation::simulate() {
    if (Np <= 0) throw std::runtime_error("no particles: call initializeParticles first");
    if (ctx) {
        slab_destroy(ctx);
        ctx = nullptr;
    }
    slab_terrain_desc td{terrain.Nx, terrain.Ny, dx, terrain.xllcorner, terrain.yllcorner};
    check(slab_create(&td, terrain.z.data(), &ctx), nullptr, "slab_create");
    slab_params p{};
    p.gravity = gravity;
    p.rho = rho;
    p.C_cfl = C_cfl;
    p.dt_max = dt_max;
    p.flip_ratio = flip_ratio;
    p.output_dt = output_dt;
    p.total_time = total_time;
    p.friction.type = (int32_t)friction.type;
    p.friction.coulomb_mu = friction.coulomb.mu;
    p.friction.voellmy_mu = friction.voellmy.mu;
    p.friction.voellmy_xi = friction.voellmy.xi;
    p.friction.mu_1 = friction.muI.mu_1;
    p.friction.mu_2 = friction.muI.mu_2;
    p.friction.I0 = friction.muI.I0;
    p.friction.d = friction.muI.d;
    p.friction.phi = friction.muI.phi;
    p.precision = (int32_t)precision;
    check(slab_set_params(ctx, &p), ctx, "slab_set_params");
    check(slab_upload_particles(ctx, Np, &particles.x[0](0), &particles.v[0](0), particles.vz.data(), particles.h.data(),
                                particles.A.data(), particles.mass.data(), particles.z.data()),
          ctx, "slab_upload_particles");
    check(slab_initial_pass(ctx), ctx, "slab_initial_pass");
    time = 0.0;
    frame = 0;
    steps = 0;
    std::unique_ptr<FrameWriter> writer;
    int64_t captured = 0;
    auto capture = [&] {
        // frame k reuses the slot of frame k - 2: its files must be written first
        writer->wait_written(captured - 2);
        check(slab_frame_capture(ctx, (int32_t)(captured % 2)), ctx, "slab_frame_capture");
        writer->push(captured++);
    };
    if (write_outputs) {
        writer.reset(new FrameWriter(ctx, [this](const slab_frame& f) {
            write_ply_vertices(particle_path / frame_name("particles_frame_", padding, f.frame, ".ply"), f.Np, f.particles);
            if (f.Nx > 0 && f.Ny > 0)
                write_grid_bands_tif(raster_path / frame_name("rasters_frame_", padding, f.frame, ".tif"), f.Nx, f.Ny, f.grid,
                                     terrain.xllcorner + terrain.x[f.i_off], terrain.yllcorner + terrain.y[f.j_off + f.Ny - 1], dx);
        }));
        capture();
    }
    while (time < total_time) {
        int64_t k = 0;
        int32_t f = frame;
        check(slab_advance_to_frame(ctx, &time, &f, &k), ctx, "slab_advance_to_frame");
        frame = f;
        steps += k;
        if (write_outputs && k > 0) capture();
        if (k == 0) break;
    }
    if (writer) {
        writer->wait_written(captured - 1);
        writer.reset();
    }
    check(slab_download_max(ctx, terrain.h_max.data(), terrain.v_max2.data()), ctx, "slab_download_max");
    pull_frame();  // the final state into particles / grid
    if (write_outputs) saveMaxData();
    std::cout << "Simulation finished: " << steps << " steps, t = " << time << " s" << std::endl;
}

// src/save_function.cpp:36-74
void Simulation::saveParticleData() const {
    write_particles_ply(particle_path / frame_name("particles_frame_", padding, frame, ".ply"), particles);
}

// src/save_function.cpp:96-226
void Simulation::saveGridData() const {
    write_grid_tif(raster_path / frame_name("rasters_frame_", padding, frame, ".tif"), grid, terrain.xllcorner, terrain.yllcorner, dx);
}

// src/save_function.cpp:228-289
void Simulation::saveMaxData() const { write_max_tif(sim_dir_path / "max_values.tif", terrain, dx); }

}  // namespace slab
