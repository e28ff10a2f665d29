// Device-side binning of a new FP32 split scenario (bin32.cu).
#pragma once

#include <vector>

#include "engine.hpp"
#include "split32.cuh"

namespace slab {

struct BinResult {
    std::vector<uint32_t> tiles;  // occupied tiles in increasing order (the first active list)
    uint64_t box_bits[4] = {0x7ff0000000000000ull, 0, 0x7ff0000000000000ull, 0};  // min x, max x, min y, max y (double bits)
    uint64_t vmax2_bits = 0;      // max |v|^2 of the FP32 velocities (double bits)
};

// Bins Np particles given as the reference's FP64 host arrays into the tile
// segments of buffer `out` (sorted by tile, upload order inside a tile), writes
// the occupied tiles' segment records (stamp 0) into grp0, the first active
// list and the active stamps. Throws SLAB_E_DOMAIN if a stencil leaves the
// terrain and SLAB_E_OOM if more than act_cap tiles are occupied.
// Its temporaries come from `scratch`.
BinResult bin_particles(const Terrain& T, int TY, int ntiles, cudaStream_t st, int Np, const double* x, const double* v, const double* vz,
                        const double* h, const double* m, const double* z, const PBuf& out, int32_t* grp0, int32_t* act_list0,
                        int32_t* act_stamp, int act_cap, Scratch& scratch);

}  // namespace slab
