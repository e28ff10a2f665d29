// PLY and GeoTIFF writers (no GDAL / tinyply). The TIFF is a classic
// little-endian TIFF 6.0 file: chunky (pixel-interleaved) float32 samples in
// strips, the floating-point predictor of Adobe's TIFF Technical Note 3 when
// compressed, and the GeoTIFF / GDAL tags that carry the geotransform, the
// nodata value and the band names.
#include "writers.hpp"

#include <dlfcn.h>
#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>

#include "slab_host.h"

namespace fs = std::filesystem;

namespace slab {

namespace {

// ---- ZSTD through the shared library, when present (no headers needed)
struct Zstd {
    using bound_fn = size_t (*)(size_t);
    using compress_fn = size_t (*)(void*, size_t, const void*, size_t, int);
    using iserr_fn = unsigned (*)(size_t);
    bound_fn bound = nullptr;
    compress_fn compress = nullptr;
    iserr_fn is_error = nullptr;
    bool ok = false;
    Zstd() {
        void* h = dlopen("libzstd.so.1", RTLD_NOW | RTLD_LOCAL);
        if (!h) return;
        bound = reinterpret_cast<bound_fn>(dlsym(h, "ZSTD_compressBound"));
        compress = reinterpret_cast<compress_fn>(dlsym(h, "ZSTD_compress"));
        is_error = reinterpret_cast<iserr_fn>(dlsym(h, "ZSTD_isError"));
        ok = bound && compress && is_error;
    }
};

const Zstd& zstd() {
    static Zstd z;
    return z;
}

// floating-point predictor of one row of n 4-byte samples (stride = samples
// per pixel): the bytes are regrouped by significance (most significant
// first), then each byte is replaced by its difference to the byte `stride`
// places before it
void fp_predict_row(const float* src, size_t n, int stride, std::vector<uint8_t>& out) {
    const size_t nb = n * 4;
    out.resize(nb);
    const uint8_t* b = reinterpret_cast<const uint8_t*>(src);
    for (size_t k = 0; k < n; ++k)
        for (int byte = 0; byte < 4; ++byte) out[(size_t)(3 - byte) * n + k] = b[4 * k + byte];  // little-endian host
    for (size_t i = nb - 1; i >= (size_t)stride; --i) out[i] = (uint8_t)(out[i] - out[i - stride]);
}

std::vector<uint8_t> compress_block(const std::vector<uint8_t>& raw, TiffCompression comp) {
    if (comp == TiffCompression::Deflate) {
        uLongf cap = compressBound((uLong)raw.size());
        std::vector<uint8_t> out(cap);
        if (compress2(out.data(), &cap, raw.data(), (uLong)raw.size(), 6) != Z_OK) throw std::runtime_error("DEFLATE failed");
        out.resize(cap);
        return out;
    }
    if (comp == TiffCompression::Zstd) {
        const Zstd& z = zstd();
        std::vector<uint8_t> out(z.bound(raw.size()));
        const size_t r = z.compress(out.data(), out.size(), raw.data(), raw.size(), 9);
        if (z.is_error(r)) throw std::runtime_error("ZSTD failed");
        out.resize(r);
        return out;
    }
    return raw;
}

struct Entry {
    uint16_t tag, type;
    uint32_t count;
    std::vector<uint8_t> data;  // value bytes (inline if <= 4)
};

enum : uint16_t { T_BYTE = 1, T_ASCII = 2, T_SHORT = 3, T_LONG = 4, T_DOUBLE = 12 };

template <typename V> Entry entry(uint16_t tag, uint16_t type, const std::vector<V>& v) {
    Entry e{tag, type, (uint32_t)v.size(), {}};
    e.data.resize(v.size() * sizeof(V));
    std::memcpy(e.data.data(), v.data(), e.data.size());
    return e;
}

Entry ascii(uint16_t tag, const std::string& s) {
    Entry e{tag, T_ASCII, (uint32_t)s.size() + 1, {}};
    e.data.assign(s.begin(), s.end());
    e.data.push_back(0);
    return e;
}

std::string xml_escape(const std::string& s) {
    std::string o;
    for (char c : s) {
        if (c == '<') o += "&lt;";
        else if (c == '>') o += "&gt;";
        else if (c == '&') o += "&amp;";
        else o += c;
    }
    return o;
}

}  // namespace

TiffCompression default_tiff_compression() { return zstd().ok ? TiffCompression::Zstd : TiffCompression::Deflate; }

void write_geotiff(const fs::path& file, int nx, int ny, const std::vector<std::vector<float>>& bands, const std::vector<std::string>& names,
                   double origin_x, double origin_y, double pixel, float nodata, TiffCompression comp) {
    const int spp = (int)bands.size();
    if (nx <= 0 || ny <= 0 || spp <= 0) throw std::runtime_error("empty raster: " + file.string());
    for (const auto& b : bands)
        if (b.size() != (size_t)nx * ny) throw std::runtime_error("band size mismatch: " + file.string());
    if (comp == TiffCompression::Zstd && !zstd().ok) comp = TiffCompression::Deflate;
    const size_t row_samples = (size_t)nx * spp;
    const int rps = (int)std::max<size_t>(1, (256u << 10) / (row_samples * 4));
    const int nstrips = (ny + rps - 1) / rps;

    std::ofstream out(file, std::ios::binary);
    if (!out) throw std::runtime_error("Could not create GeoTIFF: " + file.string());
    const uint8_t hdr[8] = {'I', 'I', 42, 0, 0, 0, 0, 0};  // IFD offset patched at the end
    out.write(reinterpret_cast<const char*>(hdr), 8);
    uint64_t pos = 8;
    std::vector<uint32_t> offs(nstrips), counts(nstrips);
    std::vector<float> row(row_samples);
    std::vector<uint8_t> raw, pred;
    for (int s = 0; s < nstrips; ++s) {
        const int r0 = s * rps, r1 = std::min(ny, r0 + rps);
        raw.clear();
        for (int r = r0; r < r1; ++r) {
            for (int x = 0; x < nx; ++x)
                for (int b = 0; b < spp; ++b) row[(size_t)x * spp + b] = bands[b][(size_t)r * nx + x];
            if (comp == TiffCompression::None) {
                const uint8_t* p = reinterpret_cast<const uint8_t*>(row.data());
                raw.insert(raw.end(), p, p + row_samples * 4);
            } else {
                fp_predict_row(row.data(), row_samples, spp, pred);
                raw.insert(raw.end(), pred.begin(), pred.end());
            }
        }
        const std::vector<uint8_t> blk = compress_block(raw, comp);
        if (pos + blk.size() > 0xFFFFFFF0ull) throw std::runtime_error("GeoTIFF larger than 4 GB: " + file.string());
        offs[s] = (uint32_t)pos;
        counts[s] = (uint32_t)blk.size();
        out.write(reinterpret_cast<const char*>(blk.data()), (std::streamsize)blk.size());
        pos += blk.size();
        if (pos & 1) {  // word-align the next item
            out.put(0);
            ++pos;
        }
    }

    std::ostringstream md;
    md << "<GDALMetadata>\n";
    for (int b = 0; b < spp && b < (int)names.size(); ++b)
        md << "  <Item name=\"DESCRIPTION\" sample=\"" << b << "\" role=\"description\">" << xml_escape(names[b]) << "</Item>\n";
    md << "</GDALMetadata>";
    std::ostringstream nd;
    nd << nodata;

    std::vector<Entry> E;
    E.push_back(entry<uint32_t>(256, T_LONG, {(uint32_t)nx}));
    E.push_back(entry<uint32_t>(257, T_LONG, {(uint32_t)ny}));
    E.push_back(entry<uint16_t>(258, T_SHORT, std::vector<uint16_t>(spp, 32)));
    E.push_back(entry<uint16_t>(259, T_SHORT, {(uint16_t)comp}));
    E.push_back(entry<uint16_t>(262, T_SHORT, {1}));
    E.push_back(entry<uint32_t>(273, T_LONG, offs));
    E.push_back(entry<uint16_t>(277, T_SHORT, {(uint16_t)spp}));
    E.push_back(entry<uint32_t>(278, T_LONG, {(uint32_t)rps}));
    E.push_back(entry<uint32_t>(279, T_LONG, counts));
    E.push_back(entry<uint16_t>(284, T_SHORT, {1}));
    if (comp != TiffCompression::None) E.push_back(entry<uint16_t>(317, T_SHORT, {3}));
    if (spp > 1) E.push_back(entry<uint16_t>(338, T_SHORT, std::vector<uint16_t>(spp - 1, 0)));
    E.push_back(entry<uint16_t>(339, T_SHORT, std::vector<uint16_t>(spp, 3)));
    E.push_back(entry<double>(33550, T_DOUBLE, {pixel, pixel, 0.0}));
    E.push_back(entry<double>(33922, T_DOUBLE, {0.0, 0.0, 0.0, origin_x, origin_y, 0.0}));
    E.push_back(entry<uint16_t>(34735, T_SHORT, {1, 1, 0, 1, 1025, 0, 1, 1}));  // GTRasterTypeGeoKey = PixelIsArea
    E.push_back(ascii(42112, md.str()));
    E.push_back(ascii(42113, nd.str()));

    // out-of-line values after the IFD
    const uint64_t ifd = pos;
    const uint64_t ifd_size = 2 + 12 * E.size() + 4;
    const uint64_t extra = ifd + ifd_size;
    std::vector<uint8_t> ifdb, tail;
    auto put16 = [](std::vector<uint8_t>& v, uint16_t x) {
        v.push_back(x & 0xFF);
        v.push_back(x >> 8);
    };
    auto put32 = [](std::vector<uint8_t>& v, uint32_t x) {
        for (int k = 0; k < 4; ++k) v.push_back((x >> (8 * k)) & 0xFF);
    };
    put16(ifdb, (uint16_t)E.size());
    for (const Entry& e : E) {
        put16(ifdb, e.tag);
        put16(ifdb, e.type);
        put32(ifdb, e.count);
        if (e.data.size() <= 4) {
            std::vector<uint8_t> v = e.data;
            v.resize(4, 0);
            ifdb.insert(ifdb.end(), v.begin(), v.end());
        } else {
            put32(ifdb, (uint32_t)(extra + tail.size()));
            tail.insert(tail.end(), e.data.begin(), e.data.end());
            if (tail.size() & 1) tail.push_back(0);
        }
    }
    put32(ifdb, 0);  // no next IFD
    if (extra + tail.size() > 0xFFFFFFF0ull) throw std::runtime_error("GeoTIFF larger than 4 GB: " + file.string());
    out.write(reinterpret_cast<const char*>(ifdb.data()), (std::streamsize)ifdb.size());
    out.write(reinterpret_cast<const char*>(tail.data()), (std::streamsize)tail.size());
    out.seekp(4);
    const uint32_t ifd32 = (uint32_t)ifd;
    const uint8_t o[4] = {(uint8_t)(ifd32 & 0xFF), (uint8_t)((ifd32 >> 8) & 0xFF), (uint8_t)((ifd32 >> 16) & 0xFF), (uint8_t)(ifd32 >> 24)};
    out.write(reinterpret_cast<const char*>(o), 4);
    if (!out) throw std::runtime_error("Failed writing GeoTIFF: " + file.string());
}

void write_ply_vertices(const fs::path& file, int n, const float* verts) {
    std::ofstream out(file, std::ios::binary);
    if (!out) throw std::runtime_error("Could not create PLY: " + file.string());
    out << "ply\nformat binary_little_endian 1.0\nelement vertex " << n << "\n";
    for (const char* name : {"x", "y", "vx", "vy", "vz", "z", "h", "A"}) out << "property float " << name << "\n";
    out << "end_header\n";
    if (n > 0) out.write(reinterpret_cast<const char*>(verts), (std::streamsize)((size_t)n * 8 * sizeof(float)));
    if (!out) throw std::runtime_error("Failed writing PLY: " + file.string());
}

void write_grid_bands_tif(const fs::path& file, int nx, int ny, const float* bands, double origin_x, double origin_y, double dx,
                          TiffCompression comp) {
    if (nx <= 0 || ny <= 0) return;
    const size_t n = (size_t)nx * ny;
    std::vector<std::vector<float>> b(6);
    for (int q = 0; q < 6; ++q) b[q].assign(bands + q * n, bands + (q + 1) * n);
    write_geotiff(file, nx, ny, b, {"h", "v_norm", "m", "v_x", "v_y", "v_z"}, origin_x, origin_y, dx, -9999.0f, comp);
}

void write_particles_ply(const fs::path& file, const Particles& p) {
    const int n = p.size();
    std::vector<float> buf((size_t)n * 8);
    for (int i = 0; i < n; ++i) {
        float* r = buf.data() + (size_t)i * 8;
        r[0] = (float)p.x[i](0);
        r[1] = (float)p.x[i](1);
        r[2] = (float)p.v[i](0);
        r[3] = (float)p.v[i](1);
        r[4] = (float)p.vz[i];
        r[5] = (float)p.z[i];
        r[6] = (float)p.h[i];
        r[7] = (float)p.A[i];
    }
    write_ply_vertices(file, n, buf.data());
}

void write_grid_tif(const fs::path& file, const Grid& g, double xll, double yll, double dx, TiffCompression comp) {
    const int nx = g.Nx, ny = g.Ny;
    if (nx <= 0 || ny <= 0) return;
    constexpr float nodata = -9999.0f;
    std::vector<std::vector<float>> b(6, std::vector<float>((size_t)nx * ny));
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const size_t k = (size_t)ind(i, j, ny), d = (size_t)(ny - 1 - j) * nx + i;
            const float hv = (float)g.h[k];
            if (hv == 0.0f) {
                for (int q = 0; q < 6; ++q) b[q][d] = nodata;
            } else {
                b[0][d] = hv;
                b[1][d] = (float)std::sqrt(g.v[k].squaredNorm());
                b[2][d] = (float)g.mass[k];
                b[3][d] = (float)g.v[k](0);
                b[4][d] = (float)g.v[k](1);
                b[5][d] = (float)g.vz[k];
            }
        }
    write_geotiff(file, nx, ny, b, {"h", "v_norm", "m", "v_x", "v_y", "v_z"}, xll + g.x.front(), yll + g.y.back(), dx, nodata, comp);
}

void write_max_tif(const fs::path& file, const Grid& t, double dx, TiffCompression comp) {
    const int nx = t.Nx, ny = t.Ny;
    constexpr float nodata = -9999.0f;
    std::vector<std::vector<float>> b(2, std::vector<float>((size_t)nx * ny));
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const size_t k = (size_t)ind(i, j, ny), d = (size_t)(ny - 1 - j) * nx + i;
            const float hv = (float)t.h_max[k];
            if (hv == 0.0f) {
                b[0][d] = b[1][d] = nodata;
            } else {
                b[0][d] = hv;
                b[1][d] = (float)std::sqrt(t.v_max2[k]);
            }
        }
    write_geotiff(file, nx, ny, b, {"h_max", "v_norm_max"}, t.xllcorner, t.yllcorner + t.y.back(), dx, nodata, comp);
}

}  // namespace slab

// ---- C entry points of the writers (include/slab_host.h)

extern "C" int slab_write_geotiff(const char* path, int32_t nx, int32_t ny, int32_t nbands, const float* bands, const char* names,
                                  double origin_x, double origin_y, double pixel, float nodata, int32_t compression) {
    try {
        if (!path || !bands || nx <= 0 || ny <= 0 || nbands <= 0) return 1;
        std::vector<std::vector<float>> b(nbands);
        for (int q = 0; q < nbands; ++q) b[q].assign(bands + (size_t)q * nx * ny, bands + (size_t)(q + 1) * nx * ny);
        std::vector<std::string> nm;
        if (names) {
            std::string cur;
            for (const char* c = names; *c; ++c) {
                if (*c == ',') {
                    nm.push_back(cur);
                    cur.clear();
                } else {
                    cur += *c;
                }
            }
            nm.push_back(cur);
        }
        const slab::TiffCompression comp =
            compression < 0 ? slab::default_tiff_compression() : static_cast<slab::TiffCompression>(compression);
        if (comp != slab::TiffCompression::None && comp != slab::TiffCompression::Deflate && comp != slab::TiffCompression::Zstd) return 1;
        slab::write_geotiff(path, nx, ny, b, nm, origin_x, origin_y, pixel, nodata, comp);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "slab_write_geotiff: %s\n", e.what());
        return 2;
    }
}

extern "C" int slab_write_ply(const char* path, int32_t n, const double* x_xy, const double* v_xy, const double* vz, const double* z,
                              const double* h, const double* A) {
    try {
        if (!path || n < 0 || (n > 0 && (!x_xy || !v_xy || !vz || !z || !h || !A))) return 1;
        slab::Particles p(n);
        for (int i = 0; i < n; ++i) {
            p.x[i] = slab::Vec2(x_xy[2 * i], x_xy[2 * i + 1]);
            p.v[i] = slab::Vec2(v_xy[2 * i], v_xy[2 * i + 1]);
            p.vz[i] = vz[i];
            p.z[i] = z[i];
            p.h[i] = h[i];
            p.A[i] = A[i];
        }
        slab::write_particles_ply(path, p);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "slab_write_ply: %s\n", e.what());
        return 2;
    }
}

extern "C" int slab_tiff_default_compression(void) { return (int)slab::default_tiff_compression(); }
