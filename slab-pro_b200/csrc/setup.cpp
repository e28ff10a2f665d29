// Host-side setup utilities exported through the C ABI.
//
// slab_poisson_disk: Bridson's Poisson-disk sampler in the form the reference
// uses for POISSON release sampling (Poisson_disk, src/poisson_disk_sampling.hpp:
// background grid of cell r/sqrt(2), k candidate points per active sample at
// distance U(r, 2r) and angle U(0, 2 pi), 21-cell neighbourhood test, uniform
// choice of the active sample, which is dropped once its k candidates fail).
// With seed 0 it draws from the C library's rand() after srand(1), which is
// the sequence the reference consumes (it never seeds, and glibc's default
// seed is 1), so the samples match the reference's. Any other seed selects a
// project-owned xorshift generator for reproducible synthetic workloads.
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <vector>

#include "slab_gpu.h"

namespace {

struct Rng {
    bool crand;
    uint64_t s;
    explicit Rng(uint64_t seed) : crand(seed == 0), s(seed * 0x9E3779B97F4A7C15ull + 1) {
        if (crand) std::srand(1);
    }
    // uniform in [0, 1] like rand()/RAND_MAX
    double unit() {
        if (crand) return static_cast<double>(std::rand()) / RAND_MAX;
        return (double)(next() >> 11) * (1.0 / 9007199254740991.0);
    }
    // uniform integer in [0, n)
    int below(int n) {
        if (crand) return std::rand() % n;
        return (int)(next() % (uint64_t)n);
    }
    uint64_t next() {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        return s;
    }
};

}  // namespace

extern "C" slab_status slab_poisson_disk(double Lx, double Ly, double r, int32_t k, uint64_t seed, double* out_xy, int64_t cap,
                                         int64_t* n_out) {
    if (!(Lx > 0) || !(Ly > 0) || !(r > 0) || k <= 0 || !n_out) return SLAB_E_ARG;
    const double a = r / std::sqrt(2);
    const int64_t Nx = static_cast<int64_t>(Lx / a) + 1, Ny = static_cast<int64_t>(Ly / a) + 1;
    if (Nx * Ny > (int64_t(1) << 33)) return SLAB_E_ARG;
    std::vector<int> cells(Nx * Ny, -1);
    std::vector<double> px, py;
    Rng rng(seed);
    auto cell_of = [&](double x, double y, int64_t& ci, int64_t& cj) {
        ci = static_cast<int64_t>(std::floor(x / a));
        cj = static_cast<int64_t>(std::floor(y / a));
    };
    static const int off[21][2] = {{-1, -2}, {0, -2}, {1, -2}, {-2, -1}, {-1, -1}, {0, -1}, {1, -1}, {2, -1}, {-2, 0}, {-1, 0}, {1, 0},
                                   {2, 0},   {-2, 1}, {-1, 1}, {0, 1},   {1, 1},   {2, 1},  {-1, 2}, {0, 2},  {1, 2},  {0, 0}};
    auto valid = [&](double x, double y) {
        int64_t ci, cj;
        cell_of(x, y, ci, cj);
        for (const auto& o : off) {
            const int64_t ni = ci + o[0], nj = cj + o[1];
            if (ni < 0 || ni >= Nx || nj < 0 || nj >= Ny) continue;
            const int s = cells[ni * Ny + nj];
            if (s < 0) continue;
            const double dx = px[s] - x, dy = py[s] - y;
            if (dx * dx + dy * dy < r * r) return false;
        }
        return true;
    };
    {
        const double x0 = rng.unit() * Lx;
        const double y0 = rng.unit() * Ly;
        px.push_back(x0);
        py.push_back(y0);
        int64_t ci, cj;
        cell_of(x0, y0, ci, cj);
        cells[ci * Ny + cj] = 0;
    }
    std::vector<int> active{0};
    int nsamples = 0;
    while (!active.empty()) {
        const int idx = rng.below(static_cast<int>(active.size()));
        const double rx = px[active[idx]], ry = py[active[idx]];
        bool found = false;
        double cx = -1, cy = -1;
        for (int t = 0; t < k; ++t) {
            const double rho = rng.unit() * r + r;
            const double theta = rng.unit() * 2 * M_PI;
            const double x = rx + rho * std::cos(theta), y = ry + rho * std::sin(theta);
            if (x >= 0 && x <= Lx && y >= 0 && y <= Ly && valid(x, y)) {
                cx = x;
                cy = y;
                found = true;
                break;
            }
        }
        if (!found) {
            active.erase(active.begin() + idx);
        } else {
            px.push_back(cx);
            py.push_back(cy);
            nsamples += 1;
            active.push_back(nsamples);
            int64_t ci, cj;
            cell_of(cx, cy, ci, cj);
            cells[ci * Ny + cj] = nsamples;
        }
    }
    const int64_t n = static_cast<int64_t>(px.size());
    *n_out = n;
    if (!out_xy) return SLAB_OK;
    if (n > cap) return SLAB_E_OOM;
    for (int64_t q = 0; q < n; ++q) {
        out_xy[2 * q] = px[q];
        out_xy[2 * q + 1] = py[q];
    }
    return SLAB_OK;
}
