// Host data containers of the simulation, laid out as the reference's
// (src/data_arrays.hpp:22-98, src/tools.hpp:27-88): per-particle vectors with
// 2-vectors stored as two contiguous doubles, node arrays flattened i * Ny + j.
// These are the arrays a caller of the step loop reads and writes; the device
// keeps its own layout and converts at upload / download.
#pragma once

#include <cmath>
#include <filesystem>
#include <string>
#include <vector>

namespace slab {

using T = double;

// 2-vector of two contiguous doubles (std::vector<Vec2> is x0, y0, x1, y1, ...)
struct Vec2 {
    double d[2] = {0.0, 0.0};
    Vec2() = default;
    Vec2(double x, double y) : d{x, y} {}
    static Vec2 Zero() { return Vec2(); }
    double& operator()(int k) { return d[k]; }
    double operator()(int k) const { return d[k]; }
    double& operator[](int k) { return d[k]; }
    double operator[](int k) const { return d[k]; }
    double squaredNorm() const { return d[0] * d[0] + d[1] * d[1]; }
    Vec2 operator+(const Vec2& o) const { return Vec2(d[0] + o.d[0], d[1] + o.d[1]); }
    Vec2 operator-(const Vec2& o) const { return Vec2(d[0] - o.d[0], d[1] - o.d[1]); }
};
static_assert(sizeof(Vec2) == 2 * sizeof(double), "Vec2 must be two packed doubles");

enum class TerrainType { Analytical, DEM };
enum class ReleaseShapeType { Rectangle, Ellipse, Polygon, Raster };
enum class SamplingMethod { Uniform, Poisson };
enum class FrictionType { Coulomb, Voellmy, mu_I };

struct Rectangle {
    Vec2 center;
    T Lx, Ly, rotation;  // rotation in radians
};
struct Ellipse {
    Vec2 center;
    T rx, ry, rotation;
};
struct Polygon {
    std::filesystem::path filepath;
    std::vector<Vec2> vertices;
};
struct Raster {
    std::filesystem::path filepath;
    T h_min = 0.0;
};
struct CoulombFriction {
    double mu;
};
struct VoellmyFriction {
    double mu, xi;
};
struct MuIFriction {
    double mu_1, mu_2, I0, d, phi;
};
struct Friction {
    FrictionType type;
    CoulombFriction coulomb;
    VoellmyFriction voellmy;
    MuIFriction muI;
};

class Particles {
  public:
    explicit Particles(int Np = 0)
        : x(Np), z(Np, 0.0), v(Np), vz(Np, 0.0), h(Np, 0.0), A(Np, 0.0), mass(Np, 0.0), theta(Np, 0.0), order(Np, 0) {}
    std::vector<Vec2> x;
    std::vector<T> z;
    std::vector<Vec2> v;
    std::vector<T> vz;
    std::vector<T> h;
    std::vector<T> A;
    std::vector<T> mass;
    std::vector<T> theta;
    std::vector<int> order;
    int size() const { return (int)h.size(); }
};

class Grid {
  public:
    explicit Grid(int Nx_in = 0, int Ny_in = 0) : Nx(Nx_in), Ny(Ny_in) { resize(Nx_in, Ny_in); }
    void resize(int nx, int ny) {
        Nx = nx;
        Ny = ny;
        const size_t n = (size_t)nx * ny;
        x.assign(nx, 0.0);
        y.assign(ny, 0.0);
        v.assign(n, Vec2());
        vz.assign(n, 0.0);
        a.assign(n, Vec2());
        mass.assign(n, 0.0);
        F.assign(n, Vec2());
        z.assign(n, 0.0);
        h.assign(n, 0.0);
        h_max.assign(n, 0.0);
        v_max2.assign(n, 0.0);
        gradients.assign(n, Vec2());
        flip.assign(n, Vec2());
        theta.assign(n, 0.0);
    }
    std::vector<T> x, y;
    std::vector<Vec2> v;
    std::vector<T> vz;
    std::vector<Vec2> a;  // F / mass, without friction
    std::vector<T> mass;
    std::vector<Vec2> F;  // P2G force sum
    std::vector<T> z;
    std::vector<T> h;
    std::vector<T> h_max;
    std::vector<T> v_max2;
    std::vector<Vec2> gradients;
    std::vector<Vec2> flip;  // v - v_old: the FLIP increment, friction included
    std::vector<T> theta;
    T xllcorner = 0.0, yllcorner = 0.0;
    int Nx = 0, Ny = 0;
    T nodata = -9999.0;
};

struct RasterData {
    std::vector<T> x, y, z;  // z[i * nrows + j], i = column (x), j = row counted from the south edge
    int ncols = 0, nrows = 0;
    T xllcorner = 0.0, yllcorner = 0.0, cellsize = 0.0, nodata = -9999.0;
};

inline int ind(int i, int j, int Ny) { return i * Ny + j; }

}  // namespace slab
