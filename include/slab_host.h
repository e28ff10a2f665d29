/* slab_host.h -- C entry points of the host library libslab_sim.so: the
 * output writers used by Simulation::saveParticleData / saveGridData /
 * saveMaxData (reference: src/save_function.cpp:36-289, which writes through
 * tinyply and GDAL). The C++ API of the same library is the Simulation class
 * in slab-pro_b200/host/simulation.hpp.
 *
 * Return value: 0 on success, 1 for invalid arguments, 2 when the file could
 * not be written (a message goes to stderr). */
#ifndef SLAB_HOST_H
#define SLAB_HOST_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* TIFF compression codes accepted by slab_write_geotiff. */
enum { SLAB_TIFF_NONE = 1, SLAB_TIFF_DEFLATE = 8, SLAB_TIFF_ZSTD = 50000 };

/* Float32 GeoTIFF of nbands bands, each nx * ny values in GDAL order (row 0
 * is the north edge, x fastest), stored pixel-interleaved. names: band
 * descriptions separated by commas (or NULL). The geotransform is
 * {origin_x, pixel, 0, origin_y, 0, -pixel}; nodata goes to GDAL's nodata
 * tag. compression: one of SLAB_TIFF_*, with the floating-point predictor
 * when compressed; -1 picks ZSTD when libzstd.so.1 can be loaded, else
 * DEFLATE -- the reference writes ZSTD with predictor 3. */
int slab_write_geotiff(const char* path, int32_t nx, int32_t ny, int32_t nbands, const float* bands, const char* names,
                       double origin_x, double origin_y, double pixel, float nodata, int32_t compression);

/* Binary little-endian PLY of n particles with float32 x y vx vy vz z h A,
 * the vertex layout of the reference's particles_frame_N.ply. */
int slab_write_ply(const char* path, int32_t n, const double* x_xy, const double* v_xy, const double* vz, const double* z,
                   const double* h, const double* A);

/* The compression -1 resolves to (SLAB_TIFF_ZSTD or SLAB_TIFF_DEFLATE). */
int slab_tiff_default_compression(void);

#ifdef __cplusplus
}
#endif

#endif
