// Release setup on the device: the particles of a RECTANGLE or ELLIPSE
// release with UNIFORM 2x2 sampling, as Simulation::initializeParticles
// builds them (src/simulation.cpp:259-476), in the reference's order and
// arithmetic. Every rounding step is written out (__dmul_rn, __dadd_rn, ...)
// so that no multiply-add is fused and the doubles equal the reference's.
// The host keeps the scalar parts the reference computes once (bounding box
// snap, cos / sin of the rotation through the C library, the sequential sum
// of h for A = V / sum h), the device does the per-sample and per-particle
// parts: the 2x2 samples of every cell, the shape filter, a stable
// compaction in sample order, and h, A, mass and the 4x4 z stencil.
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <cmath>

#include "release.hpp"

namespace slab {
namespace {

struct Shape {
    int type;
    double x_min, y_min, dx;
    int nyc;
    double cx, cy, c, s, a, b;  // c, s: cos / sin of minus the rotation
};

// sample k of the reference's loop order: cell (i, j) of the box, then the
// 2x2 displacements d (src/simulation.cpp:364-383), shifted by the box corner
__device__ __forceinline__ void sample_position(const Shape& S, int64_t k, double& x, double& y) {
    const int d = (int)(k & 3);
    const int64_t cell = k >> 2;
    const int i = (int)(cell / S.nyc), j = (int)(cell % S.nyc);
    const double dxp = (d & 1) ? 0.75 : 0.25, dyp = (d & 2) ? 0.75 : 0.25;
    const double px = __dmul_rn(__dadd_rn((double)i, dxp), S.dx), py = __dmul_rn(__dadd_rn((double)j, dyp), S.dx);
    x = __dadd_rn(px, S.x_min);
    y = __dadd_rn(py, S.y_min);
}

// the shape filter (src/simulation.cpp:398-410), rotatePoint (:478-482)
__global__ void k_release_keep(Shape S, int64_t n, unsigned char* __restrict__ keep) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double x, y;
        sample_position(S, k, x, y);
        const double p0 = __dsub_rn(x, S.cx), p1 = __dsub_rn(y, S.cy);
        const double l0 = __dsub_rn(__dmul_rn(S.c, p0), __dmul_rn(S.s, p1));
        const double l1 = __dadd_rn(__dmul_rn(S.s, p0), __dmul_rn(S.c, p1));
        bool in;
        if (S.type == SLAB_RELEASE_RECTANGLE) {
            in = fabs(l0) <= __ddiv_rn(S.a, 2.0) && fabs(l1) <= __ddiv_rn(S.b, 2.0);
        } else {
            const double u = __ddiv_rn(l0, S.a), v = __ddiv_rn(l1, S.b);
            in = __dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v)) <= 1.0;  // pow(u, 2.) + pow(v, 2.) <= 1
        }
        keep[k] = in ? 1 : 0;
    }
}

// quadratic B-spline N(u) of src/tools.hpp:119-128
__device__ __forceinline__ double Nq(double u) {
    const double a = fabs(u);
    if (a < 0.5) return __dsub_rn(0.75, __dmul_rn(a, a));
    if (a < 1.5) {
        const double r = __dsub_rn(1.5, a);
        return __dmul_rn(__dmul_rn(0.5, r), r);
    }
    return 0.0;
}

// particle p = sample sel[p]: position, h0, A, mass = rho h A, z by the 4x4
// stencil (src/simulation.cpp:433-466), v = vz = 0
__global__ void k_release_particles(Shape S, int Np, const int* __restrict__ sel, double h0, double A_init, double rho,
                                    const double* __restrict__ zt, int Nx, int Ny, double ood, ReleaseView out, int* __restrict__ err) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < Np; p += gridDim.x * blockDim.x) {
        double x, y;
        sample_position(S, sel[p], x, y);
        out.x[2 * p] = x;
        out.x[2 * p + 1] = y;
        out.v[2 * p] = 0.0;
        out.v[2 * p + 1] = 0.0;
        out.vz[p] = 0.0;
        out.h[p] = h0;
        out.A[p] = A_init;
        out.m[p] = __dmul_rn(__dmul_rn(rho, h0), A_init);
        const int ib = (int)__dmul_rn(x, ood) - 1, jb = (int)__dmul_rn(y, ood) - 1;  // terrain.x[0] = terrain.y[0] = 0
        double zp = 0.0;
        if (ib < 0 || jb < 0 || ib + 3 > Nx - 1 || jb + 3 > Ny - 1) {
            atomicOr(err, 1);
        } else {
            for (int i = ib; i < ib + 4; ++i) {
                const double xi = __dmul_rn((double)i, S.dx);
                for (int j = jb; j < jb + 4; ++j) {
                    const double yj = __dmul_rn((double)j, S.dx);
                    const double w = __dmul_rn(Nq(__dmul_rn(__dsub_rn(x, xi), ood)), Nq(__dmul_rn(__dsub_rn(y, yj), ood)));
                    zp = __dadd_rn(zp, __dmul_rn(zt[(int64_t)i * Ny + j], w));
                }
            }
        }
        out.z[p] = zp;
    }
}

}  // namespace

int64_t release_estimate(const slab_release& r, double dx) {
    const double area = r.type == SLAB_RELEASE_RECTANGLE ? r.a * r.b : M_PI * r.a * r.b;
    return (int64_t)std::ceil(area * 4.0 / (dx * dx) * 1.02) + 64;
}

DevRelease generate_release(const Terrain& T, const slab_release& r, double rho, cudaStream_t st) {
    if (r.type != SLAB_RELEASE_RECTANGLE && r.type != SLAB_RELEASE_ELLIPSE) throw Error{SLAB_E_ARG, "unknown release type"};
    if (!(r.a > 0) || !(r.b > 0) || !(r.h0 > 0) || !std::isfinite(r.cx) || !std::isfinite(r.cy) || !std::isfinite(r.rotation_deg))
        throw Error{SLAB_E_ARG, "release sizes and h0 must be > 0 and finite"};
    const double dx = T.dx, ood = 1.0 / dx;
    // bounding box and area (src/simulation.cpp:265-285), snapped to the grid (:355-358)
    double x_min, x_max, y_min, y_max, area;
    if (r.type == SLAB_RELEASE_RECTANGLE) {
        const double diag = std::sqrt(r.a * r.a + r.b * r.b) / 2.;
        x_min = r.cx - diag;
        x_max = r.cx + diag;
        y_min = r.cy - diag;
        y_max = r.cy + diag;
        area = r.a * r.b;
    } else {
        const double big = std::max(r.a, r.b);
        x_min = r.cx - big;
        x_max = r.cx + big;
        y_min = r.cy - big;
        y_max = r.cy + big;
        area = M_PI * r.a * r.b;
    }
    const double volume = area * r.h0;
    x_min = std::floor(x_min * ood) * dx;
    x_max = std::ceil(x_max * ood) * dx;
    y_min = std::floor(y_min * ood) * dx;
    y_max = std::ceil(y_max * ood) * dx;
    const int nxc = (int)std::round((x_max - x_min) * ood), nyc = (int)std::round((y_max - y_min) * ood);
    if (nxc <= 0 || nyc <= 0) throw Error{SLAB_E_ARG, "empty release"};
    const double rot = r.rotation_deg * M_PI / 180.0;
    Shape S{r.type, x_min, y_min, dx, nyc, r.cx, r.cy, std::cos(-rot), std::sin(-rot), r.a, r.b};
    const int64_t ns = (int64_t)nxc * nyc * 4;
    if (ns > INT32_MAX) throw Error{SLAB_E_ARG, "release too large"};
    dptr<unsigned char> keep = dalloc<unsigned char>(ns);
    dptr<int> sel = dalloc<int>(ns), nsel = dalloc<int>(2);
    SLAB_CUDA(cudaMemsetAsync(nsel.get(), 0, 2 * sizeof(int), st));
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((ns + 255) / 256, 148 * 16));
    k_release_keep<<<blocks, 256, 0, st>>>(S, ns, keep.get());
    SLAB_CUDA(cudaGetLastError());
    // the kept samples in sample order (a stable compaction)
    thrust::counting_iterator<int> idx(0);
    size_t tb = 0;
    SLAB_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, idx, keep.get(), sel.get(), nsel.get(), (int)ns, st));
    dptr<char> tmp = dalloc<char>(std::max<size_t>(tb, 1));
    SLAB_CUDA(cub::DeviceSelect::Flagged(tmp.get(), tb, idx, keep.get(), sel.get(), nsel.get(), (int)ns, st));
    int Np = 0;
    SLAB_CUDA(cudaMemcpyAsync(&Np, nsel.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    SLAB_CUDA(cudaStreamSynchronize(st));
    if (Np <= 0) throw Error{SLAB_E_ARG, "the release holds no sample"};
    // A = V / sum h with sum h accumulated in particle order (src/simulation.cpp:428-441)
    double sum_h = 0.0;
    for (int p = 0; p < Np; ++p) sum_h += r.h0;
    const double A_init = volume / sum_h;
    DevRelease out;
    out.Np = Np;
    out.buf = dalloc<double>((size_t)9 * Np);
    double* b = out.buf.get();
    out.x = b;
    out.v = b + 2 * (size_t)Np;
    out.vz = b + 4 * (size_t)Np;
    out.h = b + 5 * (size_t)Np;
    out.A = b + 6 * (size_t)Np;
    out.m = b + 7 * (size_t)Np;
    out.z = b + 8 * (size_t)Np;
    const ReleaseView view = out;
    k_release_particles<<<std::max(1, std::min((Np + 255) / 256, 148 * 16)), 256, 0, st>>>(S, Np, sel.get(), r.h0, A_init, rho, T.z.get(),
                                                                                          T.Nx, T.Ny, ood, view, nsel.get() + 1);
    SLAB_CUDA(cudaGetLastError());
    int err = 0;
    SLAB_CUDA(cudaMemcpyAsync(&err, nsel.get() + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    SLAB_CUDA(cudaStreamSynchronize(st));
    if (err) throw Error{SLAB_E_DOMAIN, "release reaches the terrain edge"};
    return out;
}

}  // namespace slab
