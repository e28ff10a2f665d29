// Plain single-scenario FP64 step loop (kernels P0-P5). Compiled with
// -fmad=false: every multiply and add is the IEEE operation the reference
// performs, so the only differences from the reference are the order of the
// P2G atomic sums and the last bit of CUDA's cos/atan.
//
// Layout: particles FP64 SoA in upload order; node fields dense over the
// whole terrain (i*Ny + j). The grid box of each step is the reference's
// remesh box (src/simulation.cpp:584-642) computed on the device; it bounds
// the grid-update work and the accumulator zeroing, which replaces the
// reference's per-step reallocation.
#include <algorithm>
#include <cstring>

#include "engine.hpp"
#include "moments.cuh"

namespace slab {
namespace {

struct P64 {
    double2 *x, *v;
    double *vz, *h, *A, *m, *z;
};

struct N64 {
    double *m, *px, *py, *pvz, *hm, *Fx, *Fy;  // P2G accumulators (zero between steps)
    double2 *v, *flip;                          // grid velocity and FLIP increment of the last step
    double *out_h, *out_m, *out_vz;             // normalised grid fields for output frames
    double *out_Fx, *out_Fy;                    // the P2G force sums of output frames (Grid::F)
    double *h_max, *v_max2;                     // Grid::h_max / Grid::v_max2 of the terrain
};

// position, velocity and mass of particle p, for the moments reduction
struct PlainParticle {
    const double2* x;
    const double2* v;
    const double* m;
    __device__ void operator()(int p, double& px, double& py, double& vx, double& vy, double& mass) const {
        const double2 a = x[p], b = v[p];
        px = a.x;
        py = a.y;
        vx = b.x;
        vy = b.y;
        mass = m[p];
    }
};

struct Phys {
    double g, rho, flip_ratio, one_over_dx, dx;
    int fric;
    double mu_c, mu_v, xi, mu1, mu2, I0, d, phi;
    int Nx, Ny;
};

// quadratic B-spline and derivative in the reference's form (src/tools.hpp:119-140)
__device__ __forceinline__ double Nq(double u) {
    const double a = fabs(u);
    if (a < 0.5) return 0.75 - a * a;
    if (a < 1.5) return 0.5 * (1.5 - a) * (1.5 - a);
    return 0.0;
}
__device__ __forceinline__ double dNq(double u) {
    const double a = fabs(u);
    if (a < 0.5) return -2.0 * u;
    if (a < 1.5) return u - 1.5 * (double)((0.0 < u) - (u < 0.0));
    return 0.0;
}

__device__ __forceinline__ void stencil_weights(const Phys& P, double xp, int base, double w[3], double dw[3]) {
    for (int d = 0; d < 3; ++d) {
        const double u = (xp - (double)(base + d) * P.dx) * P.one_over_dx;
        w[d] = Nq(u);
        dw[d] = dNq(u) * P.one_over_dx;
    }
}

__global__ void k64_begin(Ctl* c, int Nx, int Ny) {
    if (threadIdx.x == 0 && blockIdx.x == 0) ctl_begin(c, Nx, Ny);
}
__global__ void k64_begin_t0(Ctl* c, int Nx, int Ny) {
    if (threadIdx.x == 0 && blockIdx.x == 0) ctl_begin_t0(c, Nx, Ny);
}

// P2G (src/simulation.cpp:726-798) with atomicAdd(double) scatter. Slope
// terms of the particle's containing cell (src/complex_terrain.cpp:113-130).
__global__ void __launch_bounds__(256) k64_p2g(const Ctl* __restrict__ c, P64 p, N64 n, const double2* __restrict__ grad,
                                               const double* __restrict__ cos_t, Phys P, int Np) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= Np || !c->active) return;
    const double2 x = p.x[q], v = p.v[q];
    const double h = p.h[q], A = p.A[q], m = p.m[q];
    const double vmx = v.x * m, vmy = v.y * m;
    const double vzm = p.vz[q] * m, hm = h * m, hA = h * A;
    const int ib = (int)floor(x.x * P.one_over_dx - 0.5), jb = (int)floor(x.y * P.one_over_dx - 0.5);
    const int cell = (int)floor(x.x * P.one_over_dx) * P.Ny + (int)floor(x.y * P.one_over_dx);
    const double2 gr = grad[cell];
    const double ct = cos_t[cell];
    const double coeff = -m * P.g * ct * ct;
    const double mbx = coeff * gr.x, mby = coeff * gr.y;
    const double s00 = -0.5 * P.rho * P.g * ct * ct * h;
    double wx[3], wy[3], dwx[3], dwy[3];
    stencil_weights(P, x.x, ib, wx, dwx);
    stencil_weights(P, x.y, jb, wy, dwy);
#pragma unroll
    for (int di = 0; di < 3; ++di) {
#pragma unroll
        for (int dj = 0; dj < 3; ++dj) {
            const double w = wx[di] * wy[dj];
            if (w > 3e-3) {
                const double gwx = dwx[di] * wy[dj], gwy = dwy[dj] * wx[di];
                const int64_t k = (int64_t)(ib + di) * P.Ny + (jb + dj);
                atomicAdd(n.m + k, m * w);
                atomicAdd(n.px + k, vmx * w);
                atomicAdd(n.py + k, vmy * w);
                atomicAdd(n.pvz + k, vzm * w);
                atomicAdd(n.hm + k, hm * w);
                atomicAdd(n.Fx + k, mbx * w - hA * (s00 * gwx + 0.0 * gwy));
                atomicAdd(n.Fy + k, mby * w - hA * (s00 * gwy + 0.0 * gwx));
            }
        }
    }
}

// Frame packing (slab_frame_capture): particle q as float32 vertex q, x y vx
// vy vz z h A (the PLY vertex layout).
__global__ void k64_pack_particles(P64 p, int Np, float* __restrict__ out) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < Np; q += gridDim.x * blockDim.x) {
        const double2 x = p.x[q], v = p.v[q];
        float* o = out + (size_t)q * 8;
        o[0] = (float)x.x;
        o[1] = (float)x.y;
        o[2] = (float)v.x;
        o[3] = (float)v.y;
        o[4] = (float)p.vz[q];
        o[5] = (float)p.z[q];
        o[6] = (float)p.h[q];
        o[7] = (float)p.A[q];
    }
}

// The grid box's 6 GeoTIFF bands (h, |v|, m, vx, vy, vz): band-major, row 0
// = the north edge, x fastest, -9999 in every band where h == 0.
__global__ void k64_pack_grid(N64 n, int Ny, int i0, int j0, int nI, int nJ, float* __restrict__ out) {
    const int64_t total = (int64_t)nI * nJ;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(k / nI), ci = (int)(k % nI);
        const int64_t g = (int64_t)(i0 + ci) * Ny + (j0 + nJ - 1 - r);
        const float h = (float)n.out_h[g];
        if (h == 0.f) {
            for (int q = 0; q < 6; ++q) out[q * total + k] = -9999.f;
            continue;
        }
        const double2 v = n.v[g];
        out[k] = h;
        out[total + k] = (float)sqrt(v.x * v.x + v.y * v.y);
        out[2 * total + k] = (float)n.out_m[g];
        out[3 * total + k] = (float)v.x;
        out[4 * total + k] = (float)v.y;
        out[5 * total + k] = (float)n.out_vz[g];
    }
}

// computeGridVelocity (src/simulation.cpp:800-875) over the remesh box, then
// the accumulators are zeroed for the next step.
__global__ void __launch_bounds__(256) k64_grid(Ctl* c, N64 n, const double2* __restrict__ grad,
                                                const double* __restrict__ cos_t, Phys P) {
    if (!c->active) return;
    const int i0 = c->box[0], j0 = c->box[2];
    const int nI = c->box[1] - i0 + 1, nJ = c->box[3] - j0 + 1;
    const int64_t total = (int64_t)nI * nJ;
    const double dt = c->dt;
    const bool outs = c->write_outputs;
    unsigned nact = 0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int i = i0 + (int)(t / nJ), j = j0 + (int)(t % nJ);
        const int64_t k = (int64_t)i * P.Ny + j;
        const double mi = n.m[k];
        double2 nv = make_double2(0.0, 0.0), fl = make_double2(0.0, 0.0);
        double hn = 0.0, vzn = 0.0;
        if (mi > 1e-6) {
            const double vox = n.px[k] / mi, voy = n.py[k] / mi;
            vzn = n.pvz[k] / mi;
            hn = n.hm[k] / mi;
            const double ax = n.Fx[k] / mi, ay = n.Fy[k] / mi;
            const double vtx = vox + dt * ax, vty = voy + dt * ay;
            const double vsq = vtx * vtx + vty * vty;
            if (vsq > 1e-16) {
                const double2 gr = grad[k];
                const double ct = cos_t[k];
                const double vz = vtx * gr.x + vty * gr.y;
                const double v3sq = vsq + vz * vz;
                const double v3 = sqrt(v3sq);
                double af;
                if (P.fric == SLAB_COULOMB) {
                    af = P.mu_c * P.g * ct;
                } else if (P.fric == SLAB_VOELLMY) {
                    af = P.mu_v * P.g * ct + P.g * v3sq / (P.xi * hn * ct);
                } else {
                    const double I = 5. * P.d * v3 / (2. * hn * ct * ct * sqrt(P.g * hn * P.phi));
                    const double muI = P.mu1 + (P.mu2 - P.mu1) / (1. + P.I0 / I);
                    af = muI * P.g * ct;
                }
                const double dv = dt * af;
                if (dv < v3) {
                    const double f = 1. - dv / v3;
                    nv = make_double2(vtx * f, vty * f);
                }
            }
            fl = make_double2(nv.x - vox, nv.y - voy);
            ++nact;
            if (n.h_max[k] < hn) n.h_max[k] = hn;
            const double v2 = nv.x * nv.x + nv.y * nv.y;
            if (n.v_max2[k] < v2) n.v_max2[k] = v2;
        }
        n.v[k] = nv;
        n.flip[k] = fl;
        if (outs) {
            n.out_h[k] = hn;
            n.out_m[k] = mi;
            n.out_vz[k] = vzn;
            n.out_Fx[k] = n.Fx[k];
            n.out_Fy[k] = n.Fy[k];
        }
        n.m[k] = 0.0;
        n.px[k] = 0.0;
        n.py[k] = 0.0;
        n.pvz[k] = 0.0;
        n.hm[k] = 0.0;
        n.Fx[k] = 0.0;
        n.Fy[k] = 0.0;
    }
    for (int o = 16; o > 0; o >>= 1) nact += __shfl_xor_sync(0xffffffffu, nact, o);
    if ((threadIdx.x & 31) == 0 && nact) atomicAdd(&c->node_steps, (unsigned long long)nact);
}

__device__ __forceinline__ uint64_t dbits(double v) { return (uint64_t)__double_as_longlong(v); }

// Block-reduce the particle bounding box and max |v|^2 into the control
// block; the last block to finish closes the step.
__device__ void block_epilogue(Ctl* c, bool valid, double px, double py, double v2, bool close_step) {
    __shared__ double s_red[5][8];
    double mnx = valid ? px : INFINITY, mxx = valid ? px : 0.0, mny = valid ? py : INFINITY, mxy = valid ? py : 0.0;
    double vv = valid ? v2 : 0.0;
    mnx = warp_min(mnx);
    mxx = warp_max(mxx);
    mny = warp_min(mny);
    mxy = warp_max(mxy);
    vv = warp_max(vv);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) {
        s_red[0][wid] = mnx;
        s_red[1][wid] = mxx;
        s_red[2][wid] = mny;
        s_red[3][wid] = mxy;
        s_red[4][wid] = vv;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < nw; ++w) {
            mnx = fmin(mnx, s_red[0][w]);
            mxx = fmax(mxx, s_red[1][w]);
            mny = fmin(mny, s_red[2][w]);
            mxy = fmax(mxy, s_red[3][w]);
            vv = fmax(vv, s_red[4][w]);
        }
        atomicMin(reinterpret_cast<unsigned long long*>(&c->pos_acc[0]), (unsigned long long)dbits(mnx));
        atomicMax(reinterpret_cast<unsigned long long*>(&c->pos_acc[1]), (unsigned long long)dbits(mxx));
        atomicMin(reinterpret_cast<unsigned long long*>(&c->pos_acc[2]), (unsigned long long)dbits(mny));
        atomicMax(reinterpret_cast<unsigned long long*>(&c->pos_acc[3]), (unsigned long long)dbits(mxy));
        atomicMax(reinterpret_cast<unsigned long long*>(&c->vmax2_acc), (unsigned long long)dbits(vv));
        if (close_step) {
            __threadfence();
            const unsigned prev = atomicAdd(&c->done_blocks, 1u);
            if (prev == gridDim.x - 1) {
                __threadfence();
                ctl_end(c);
            }
        }
    }
}

// G2P (src/simulation.cpp:877-940).
__global__ void __launch_bounds__(256) k64_g2p(Ctl* c, P64 p, N64 n, const double2* __restrict__ grad, const double* __restrict__ z,
                                               Phys P, int Np) {
    if (!c->active) return;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = q < Np;
    double2 nx = make_double2(0, 0);
    double v2 = 0.0;
    if (valid) {
        const double2 x = p.x[q];
        const int cell = (int)floor(x.x * P.one_over_dx) * P.Ny + (int)floor(x.y * P.one_over_dx);
        const double2 pg = grad[cell];
        const int ib = (int)floor(x.x * P.one_over_dx - 0.5), jb = (int)floor(x.y * P.one_over_dx - 0.5);
        double wx[3], wy[3], dwx[3], dwy[3];
        stencil_weights(P, x.x, ib, wx, dwx);
        stencil_weights(P, x.y, jb, wy, dwy);
        double picx = 0.0, picy = 0.0, flx = 0.0, fly = 0.0, zp = 0.0, strain = 0.0;
#pragma unroll
        for (int di = 0; di < 3; ++di) {
#pragma unroll
            for (int dj = 0; dj < 3; ++dj) {
                const double w = wx[di] * wy[dj];
                const int64_t k = (int64_t)(ib + di) * P.Ny + (jb + dj);
                const double gwx = dwx[di] * wy[dj], gwy = dwy[dj] * wx[di];
                const double2 gv = n.v[k], gf = n.flip[k];
                picx += gv.x * w;
                picy += gv.y * w;
                flx += gf.x * w;
                fly += gf.y * w;
                zp += z[k] * w;
                strain += gwx * gv.x + gwy * gv.y;
            }
        }
        const double dt = c->dt;
        strain *= dt;
        const double2 v = p.v[q];
        const double fr = P.flip_ratio;
        const double nvx = fr * (v.x + flx) + (1. - fr) * picx;
        const double nvy = fr * (v.y + fly) + (1. - fr) * picy;
        p.z[q] = zp;
        p.v[q] = make_double2(nvx, nvy);
        p.vz[q] = nvx * pg.x + nvy * pg.y;
        nx = make_double2(x.x + dt * picx, x.y + dt * picy);
        p.x[q] = nx;
        const double hn = p.h[q] / (1. + strain);
        p.h[q] = hn;
        p.A[q] = p.m[q] / (hn * P.rho);
        v2 = nvx * nvx + nvy * nvy;
        if (!isfinite(nx.x) || !isfinite(nx.y) || !isfinite(v2) || !isfinite(hn)) atomicOr(&c->err, ERR_NONFINITE);
        if (nx.x < 0.0 || nx.y < 0.0) atomicOr(&c->err, ERR_DOMAIN);
    }
    block_epilogue(c, valid, nx.x, nx.y, v2, true);
}

// Particle box and max |v|^2 of freshly uploaded particles.
__global__ void k64_stats(Ctl* c, P64 p, int Np) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = q < Np;
    double2 x = make_double2(0, 0);
    double v2 = 0;
    if (valid) {
        x = p.x[q];
        const double2 v = p.v[q];
        v2 = v.x * v.x + v.y * v.y;
        if (x.x < 0.0 || x.y < 0.0) atomicOr(&c->err, ERR_DOMAIN);
    }
    block_epilogue(c, valid, x.x, x.y, v2, false);
}

struct Plain64 final : Path {
    const Terrain& T;
    slab_params prm;
    cudaStream_t st;
    Ctl* dc;
    Ctl* hc;
    Phys P{};
    int Np = 0;
    dptr<double2> x, v;
    dptr<double> vz, h, A, m, z;
    dptr<double> acc;  // 7 accumulators, each Nx*Ny
    dptr<double2> gv, gflip;
    dptr<double> out5;  // out_h, out_m, out_vz, out_Fx, out_Fy
    dptr<double> maxes; // h_max, v_max2
    int64_t nlaunch = 0;
    StepGraphs graphs;
    PhaseTimer timer;

    Plain64(const Terrain& t, const slab_params& p, cudaStream_t s, Ctl* d, Ctl* h_) : T(t), prm(p), st(s), dc(d), hc(h_) {
        P.g = p.gravity;
        P.rho = p.rho;
        P.flip_ratio = p.flip_ratio;
        P.one_over_dx = 1. / t.dx;
        P.dx = t.dx;
        P.fric = p.friction.type;
        P.mu_c = p.friction.coulomb_mu;
        P.mu_v = p.friction.voellmy_mu;
        P.xi = p.friction.voellmy_xi;
        P.mu1 = p.friction.mu_1;
        P.mu2 = p.friction.mu_2;
        P.I0 = p.friction.I0;
        P.d = p.friction.d;
        P.phi = p.friction.phi;
        P.Nx = t.Nx;
        P.Ny = t.Ny;
        const size_t nn = (size_t)t.Nx * t.Ny;
        acc = dalloc<double>(7 * nn);
        gv = dalloc<double2>(nn);
        gflip = dalloc<double2>(nn);
        out5 = dalloc<double>(5 * nn);
        maxes = dalloc<double>(2 * nn);
        SLAB_CUDA(cudaMemsetAsync(acc.get(), 0, 7 * nn * sizeof(double), st));
        SLAB_CUDA(cudaMemsetAsync(gv.get(), 0, nn * sizeof(double2), st));
        SLAB_CUDA(cudaMemsetAsync(gflip.get(), 0, nn * sizeof(double2), st));
        SLAB_CUDA(cudaMemsetAsync(out5.get(), 0, 5 * nn * sizeof(double), st));
        SLAB_CUDA(cudaMemsetAsync(maxes.get(), 0, 2 * nn * sizeof(double), st));
    }

    P64 parts() { return P64{x.get(), v.get(), vz.get(), h.get(), A.get(), m.get(), z.get()}; }
    N64 nodes() {
        const size_t nn = (size_t)T.Nx * T.Ny;
        double* a = acc.get();
        double* o = out5.get();
        return N64{a, a + nn, a + 2 * nn, a + 3 * nn, a + 4 * nn, a + 5 * nn, a + 6 * nn, gv.get(), gflip.get(),
                   o, o + nn, o + 2 * nn, o + 3 * nn, o + 4 * nn, maxes.get(), maxes.get() + nn};
    }

    void upload(int np, const double* hx, const double* hv, const double* hvz, const double* hh, const double* hA, const double* hm,
                const double* hz) override {
        Np = np;
        x = dalloc<double2>(np);
        v = dalloc<double2>(np);
        vz = dalloc<double>(np);
        h = dalloc<double>(np);
        A = dalloc<double>(np);
        m = dalloc<double>(np);
        z = dalloc<double>(np);
        // host arrays, or device arrays of a release generated on the device
        SLAB_CUDA(cudaMemcpyAsync(x.get(), hx, np * sizeof(double2), cudaMemcpyDefault, st));
        SLAB_CUDA(cudaMemcpyAsync(v.get(), hv, np * sizeof(double2), cudaMemcpyDefault, st));
        SLAB_CUDA(cudaMemcpyAsync(vz.get(), hvz, np * sizeof(double), cudaMemcpyDefault, st));
        SLAB_CUDA(cudaMemcpyAsync(h.get(), hh, np * sizeof(double), cudaMemcpyDefault, st));
        SLAB_CUDA(cudaMemcpyAsync(A.get(), hA, np * sizeof(double), cudaMemcpyDefault, st));
        SLAB_CUDA(cudaMemcpyAsync(m.get(), hm, np * sizeof(double), cudaMemcpyDefault, st));
        SLAB_CUDA(cudaMemcpyAsync(z.get(), hz, np * sizeof(double), cudaMemcpyDefault, st));
        // the control block was reset by the caller; collect the initial box / max speed
        k64_stats<<<(np + 255) / 256, 256, 0, st>>>(dc, parts(), np);
        SLAB_CUDA(cudaGetLastError());
        ++nlaunch;
        SLAB_CUDA(cudaMemcpyAsync(&dc->vmax2_bits, &dc->vmax2_acc, sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
        graphs.clear();
    }

    int grid_blocks() const { return 148 * 4; }

    void launch_kernel(int k) {
        const int pb = (Np + 255) / 256;
        switch (k) {
            case 0: k64_begin<<<1, 32, 0, st>>>(dc, T.Nx, T.Ny); break;
            case 1: k64_p2g<<<pb, 256, 0, st>>>(dc, parts(), nodes(), T.grad.get(), T.cos_t.get(), P, Np); break;
            case 2: k64_grid<<<grid_blocks(), 256, 0, st>>>(dc, nodes(), T.grad.get(), T.cos_t.get(), P); break;
            case 3: k64_g2p<<<pb, 256, 0, st>>>(dc, parts(), nodes(), T.grad.get(), T.z.get(), P, Np); break;
        }
    }
    void launch_step() {
        for (int k = 0; k < 4; ++k) launch_kernel(k);
    }

    void initial_pass() override {
        k64_begin_t0<<<1, 32, 0, st>>>(dc, T.Nx, T.Ny);
        k64_p2g<<<(Np + 255) / 256, 256, 0, st>>>(dc, parts(), nodes(), T.grad.get(), T.cos_t.get(), P, Np);
        k64_grid<<<grid_blocks(), 256, 0, st>>>(dc, nodes(), T.grad.get(), T.cos_t.get(), P);
        SLAB_CUDA(cudaGetLastError());
        nlaunch += 3;
    }

    void enqueue_steps(int chunk) override {
        if (timer.on) {
            for (int k = 0; k < chunk; ++k) timer.profiled_step(st, [&](int kk) { launch_kernel(kk); });
            SLAB_CUDA(cudaGetLastError());
        } else {
            graphs.launch(chunk, st, [&] { launch_step(); });
        }
        nlaunch += 4 * chunk;
    }
    void set_profiling(bool on) override {
        timer.collect();
        timer.reset();
        timer.on = on;
    }
    void phase_times(double out[5]) override {
        timer.collect();
        for (int k = 0; k < 5; ++k) out[k] = timer.acc[k];
    }

    void download_particles(double* hx, double* hv, double* hvz, double* hh, double* hA, double* hm, double* hz) override {
        auto cp = [&](double* dst, const void* src, size_t bytes) {
            if (dst) SLAB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
        };
        cp(hx, x.get(), Np * sizeof(double2));
        cp(hv, v.get(), Np * sizeof(double2));
        cp(hvz, vz.get(), Np * sizeof(double));
        cp(hh, h.get(), Np * sizeof(double));
        cp(hA, A.get(), Np * sizeof(double));
        cp(hm, m.get(), Np * sizeof(double));
        cp(hz, z.get(), Np * sizeof(double));
        SLAB_CUDA(cudaStreamSynchronize(st));
    }

    void download_grid(slab_grid_view* gv_) override {
        SLAB_CUDA(cudaMemcpyAsync(hc, dc, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
        SLAB_CUDA(cudaStreamSynchronize(st));
        const int i0 = hc->box[0], i1 = hc->box[1], j0 = hc->box[2], j1 = hc->box[3];
        const int gNx = i1 - i0 + 1, gNy = j1 - j0 + 1;
        gv_->Nx = gNx;
        gv_->Ny = gNy;
        gv_->i_off = i0;
        gv_->j_off = j0;
        if (!grid_view_wants_fields(*gv_)) return;  // box only
        if ((int64_t)gNx * gNy > gv_->cap_nodes) throw Error{SLAB_E_ARG, "grid view capacity too small"};
        N64 n = nodes();
        // Grid::a = F / mass needs both, whichever of them the caller asked for
        std::vector<double> Fh, mh;
        double* Fdst = gv_->F;
        double* mdst = gv_->mass;
        if (gv_->a && !Fdst) {
            Fh.resize(2 * (size_t)gNx * gNy);
            Fdst = Fh.data();
        }
        if (gv_->a && !mdst) {
            mh.resize((size_t)gNx * gNy);
            mdst = mh.data();
        }
        std::vector<double> fy;
        if (Fdst) fy.resize((size_t)gNx * gNy);
        for (int i = 0; i < gNx; ++i) {
            const size_t src = (size_t)(i0 + i) * T.Ny + j0, dst = (size_t)i * gNy;
            if (gv_->h) SLAB_CUDA(cudaMemcpyAsync(gv_->h + dst, n.out_h + src, gNy * sizeof(double), cudaMemcpyDeviceToHost, st));
            if (mdst) SLAB_CUDA(cudaMemcpyAsync(mdst + dst, n.out_m + src, gNy * sizeof(double), cudaMemcpyDeviceToHost, st));
            if (gv_->vz) SLAB_CUDA(cudaMemcpyAsync(gv_->vz + dst, n.out_vz + src, gNy * sizeof(double), cudaMemcpyDeviceToHost, st));
            if (gv_->v) SLAB_CUDA(cudaMemcpyAsync(gv_->v + 2 * dst, n.v + src, gNy * sizeof(double2), cudaMemcpyDeviceToHost, st));
            if (gv_->flip) SLAB_CUDA(cudaMemcpyAsync(gv_->flip + 2 * dst, n.flip + src, gNy * sizeof(double2), cudaMemcpyDeviceToHost, st));
            if (Fdst) {  // x components into place, y components beside them, interleaved below
                SLAB_CUDA(cudaMemcpyAsync(Fdst + dst, n.out_Fx + src, gNy * sizeof(double), cudaMemcpyDeviceToHost, st));
                SLAB_CUDA(cudaMemcpyAsync(fy.data() + dst, n.out_Fy + src, gNy * sizeof(double), cudaMemcpyDeviceToHost, st));
            }
        }
        SLAB_CUDA(cudaStreamSynchronize(st));
        const size_t nn = (size_t)gNx * gNy;
        if (Fdst) {
            for (size_t k = nn; k-- > 0;) {
                Fdst[2 * k] = Fdst[k];
                Fdst[2 * k + 1] = fy[k];
            }
        }
        if (gv_->a) fill_grid_acceleration(gv_->a, Fdst, mdst, nn);
    }

    void download_max(double* hmax, double* vmax2) override {
        const size_t nn = (size_t)T.Nx * T.Ny;
        if (hmax) SLAB_CUDA(cudaMemcpyAsync(hmax, maxes.get(), nn * sizeof(double), cudaMemcpyDeviceToHost, st));
        if (vmax2) SLAB_CUDA(cudaMemcpyAsync(vmax2, maxes.get() + nn, nn * sizeof(double), cudaMemcpyDeviceToHost, st));
        SLAB_CUDA(cudaStreamSynchronize(st));
    }

    void conservation(double out[4]) override {
        std::vector<double> hmass(Np), hv(2 * (size_t)Np);
        download_particles(nullptr, hv.data(), nullptr, nullptr, nullptr, hmass.data(), nullptr);
        double M = 0, Px = 0, Py = 0;
        for (int q = 0; q < Np; ++q) {
            M += hmass[q];
            Px += hmass[q] * hv[2 * q];
            Py += hmass[q] * hv[2 * q + 1];
        }
        SLAB_CUDA(cudaMemcpyAsync(hc, dc, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
        SLAB_CUDA(cudaStreamSynchronize(st));
        const int i0 = hc->box[0], i1 = hc->box[1], j0 = hc->box[2], j1 = hc->box[3];
        double G = 0;
        std::vector<double> row(j1 - j0 + 1);
        for (int i = i0; i <= i1; ++i) {
            SLAB_CUDA(cudaMemcpy(row.data(), nodes().out_m + (size_t)i * T.Ny + j0, row.size() * sizeof(double), cudaMemcpyDeviceToHost));
            for (double r : row) G += r;
        }
        out[0] = M;
        out[1] = G;
        out[2] = Px;
        out[3] = Py;
    }

    void pack_frame(float* d_part, float* d_grid, const int32_t box[4]) override {
        k64_pack_particles<<<std::max(1, std::min(148 * 8, (Np + 255) / 256)), 256, 0, st>>>(parts(), Np, d_part);
        const int nI = box[1] - box[0] + 1, nJ = box[3] - box[2] + 1;
        const int64_t nn = (int64_t)nI * nJ;
        if (nn > 0)
            k64_pack_grid<<<(int)std::max<int64_t>(1, std::min<int64_t>((nn + 255) / 256, 148 * 8)), 256, 0, st>>>(
                nodes(), T.Ny, box[0], box[2], nI, nJ, d_grid);
        nlaunch += nn > 0 ? 2 : 1;
        SLAB_CUDA(cudaGetLastError());
    }

    dptr<double> mom;
    void moments(double out[6]) override {
        if (!mom) mom = dalloc<double>((size_t)MOM_BLOCKS * MOM_N + MOM_N);
        k_moments<<<MOM_BLOCKS, MOM_THREADS, 0, st>>>(Np, PlainParticle{x.get(), v.get(), m.get()}, mom.get());
        k_moments_final<<<1, MOM_THREADS, 0, st>>>(mom.get(), mom.get() + (size_t)MOM_BLOCKS * MOM_N);
        nlaunch += 2;
        SLAB_CUDA(cudaGetLastError());
        SLAB_CUDA(cudaMemcpyAsync(out, mom.get() + (size_t)MOM_BLOCKS * MOM_N, MOM_N * sizeof(double), cudaMemcpyDeviceToHost, st));
        SLAB_CUDA(cudaStreamSynchronize(st));
    }

    int64_t launches() const override { return nlaunch; }
};

}  // namespace

std::unique_ptr<Path> make_plain64(const Terrain& t, const slab_params& p, cudaStream_t s, Ctl* d_ctl, Ctl* h_ctl) {
    return std::unique_ptr<Path>(new Plain64(t, p, s, d_ctl, h_ctl));
}

}  // namespace slab
