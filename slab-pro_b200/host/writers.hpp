// Output files of the simulation, written without GDAL or tinyply:
//  - particles_frame_N.ply: binary little-endian PLY, one vertex element
//    with float32 x y vx vy vz z h A (src/save_function.cpp:36-74);
//  - rasters_frame_N.tif: 6-band float32 GeoTIFF h, v_norm, m, v_x, v_y,
//    v_z over the frame's grid box, nodata -9999 where h == 0
//    (src/save_function.cpp:96-226);
//  - max_values.tif: 2-band float32 GeoTIFF h_max, v_norm_max over the whole
//    terrain (src/save_function.cpp:228-289).
// GeoTIFFs carry the geotransform (pixel scale + tie point), GDAL's nodata
// and band-description tags, and are compressed like the reference's
// (ZSTD with the floating-point predictor) when libzstd can be loaded,
// else with DEFLATE and the same predictor.
#pragma once

#include <cstdint>
#include <filesystem>
#include <string>
#include <vector>

#include "data_arrays.hpp"

namespace slab {

enum class TiffCompression { None = 1, Deflate = 8, Zstd = 50000 };

// Compression used when none is asked for: ZSTD if libzstd.so.1 loads, else DEFLATE.
TiffCompression default_tiff_compression();

// Bands are nx * ny float32 in GDAL order (row 0 = north edge, x fastest).
// origin_x / origin_y: coordinates of the top-left corner; pixel: cell size.
void write_geotiff(const std::filesystem::path& file, int nx, int ny, const std::vector<std::vector<float>>& bands,
                   const std::vector<std::string>& names, double origin_x, double origin_y, double pixel, float nodata,
                   TiffCompression comp);

void write_particles_ply(const std::filesystem::path& file, const Particles& p);
// n vertices of 8 float32 (x y vx vy vz z h A), as packed by slab_frame_capture
void write_ply_vertices(const std::filesystem::path& file, int n, const float* verts);
// the 6 bands of rasters_frame_N.tif (h, v_norm, m, v_x, v_y, v_z), already in
// GDAL order with nodata -9999, as packed by slab_frame_capture
void write_grid_bands_tif(const std::filesystem::path& file, int nx, int ny, const float* bands, double origin_x, double origin_y, double dx,
                          TiffCompression comp = default_tiff_compression());
void write_grid_tif(const std::filesystem::path& file, const Grid& grid, double xll, double yll, double dx,
                    TiffCompression comp = default_tiff_compression());
void write_max_tif(const std::filesystem::path& file, const Grid& terrain, double dx, TiffCompression comp = default_tiff_compression());

}  // namespace slab
