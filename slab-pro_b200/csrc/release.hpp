// Release setup on the device (release.cu).
#pragma once

#include "engine.hpp"

namespace slab {

// device arrays of a generated particle set, in the layouts of
// slab_upload_particles (x, v interleaved)
struct ReleaseView {
    double *x, *v, *vz, *h, *A, *m, *z;
};

struct DevRelease : ReleaseView {
    int Np = 0;
    dptr<double> buf;
};

// The particles of a RECTANGLE / ELLIPSE release with UNIFORM 2x2 sampling,
// built on the device exactly as Simulation::initializeParticles builds them
// (src/simulation.cpp:259-476). Throws SLAB_E_ARG for an invalid release,
// SLAB_E_DOMAIN if its 4x4 z stencil leaves the terrain.
DevRelease generate_release(const Terrain& T, const slab_release& r, double rho, cudaStream_t st);

// An upper estimate of the release's particle count (admission before the
// particles exist): 4 per cell of its area, plus a margin.
int64_t release_estimate(const slab_release& r, double dx);

}  // namespace slab
