// Preview helpers on the host (src/render.rs): the slice-plane constructors,
// the pixel primitives (disk, Bresenham line), render_timeseries and PNG
// output. The slice image itself is drawn on the device (render.cuh); the
// needle overlay uses the primitives here.
#include <zlib.h>

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "sdr_gpu.h"

void sdr_internal_set_error(const std::string& msg);

namespace {

void put_px(uint8_t* rgb, uint32_t w, uint32_t h, int64_t x, int64_t y, const uint8_t c[3]) {  // render.rs:430-434
    if (x >= 0 && y >= 0 && (uint64_t)x < w && (uint64_t)y < h) std::memcpy(rgb + 3 * ((size_t)y * w + x), c, 3);
}

int64_t as_i64(double f) {  // Rust `as i64`
    if (std::isnan(f)) return 0;
    if (f >= 9223372036854775807.0) return INT64_MAX;
    if (f <= -9223372036854775808.0) return INT64_MIN;
    return (int64_t)f;
}

void be32(std::vector<uint8_t>& o, uint32_t v) {
    o.push_back((uint8_t)(v >> 24));
    o.push_back((uint8_t)(v >> 16));
    o.push_back((uint8_t)(v >> 8));
    o.push_back((uint8_t)v);
}

void png_chunk(std::vector<uint8_t>& o, const char* type, const uint8_t* data, size_t n) {
    be32(o, (uint32_t)n);
    size_t at = o.size();
    o.insert(o.end(), type, type + 4);
    if (n) o.insert(o.end(), data, data + n);
    uLong crc = crc32(0L, Z_NULL, 0);
    crc = crc32(crc, o.data() + at, (uInt)(n + 4));
    be32(o, (uint32_t)crc);
}

}  // namespace

void sdr_internal_draw_disk(uint8_t* rgb, uint32_t w, uint32_t h, int64_t cx, int64_t cy, int64_t r,
                            const uint8_t c[3]) {  // draw_disk, render.rs:436-444
    for (int64_t dy = -r; dy <= r; ++dy)
        for (int64_t dx = -r; dx <= r; ++dx)
            if (dx * dx + dy * dy <= r * r) put_px(rgb, w, h, cx + dx, cy + dy, c);
}

void sdr_internal_draw_line(uint8_t* rgb, uint32_t w, uint32_t h, int64_t x0, int64_t y0, int64_t x1, int64_t y1,
                            const uint8_t c[3]) {  // Bresenham, render.rs:447-468
    const int64_t dx = x1 >= x0 ? x1 - x0 : x0 - x1;
    const int64_t dy = -(y1 >= y0 ? y1 - y0 : y0 - y1);
    const int64_t sx = x0 < x1 ? 1 : -1, sy = y0 < y1 ? 1 : -1;
    int64_t err = dx + dy;
    for (;;) {
        put_px(rgb, w, h, x0, y0, c);
        if (x0 == x1 && y0 == y1) break;
        const int64_t e2 = 2 * err;
        if (e2 >= dy) {
            err += dy;
            x0 += sx;
        }
        if (e2 <= dx) {
            err += dx;
            y0 += sy;
        }
    }
}

extern "C" {

int sdr_slice_plane_xy(double slice, double slab, sdr_slice_plane* out) {  // SlicePlane::xy, render.rs:64-75
    if (!out) {
        sdr_internal_set_error("null argument");
        return SDR_ERR_INVALID;
    }
    *out = sdr_slice_plane{0, 1, 2, 1, 0, 0, slice, slab};
    return SDR_OK;
}

int sdr_slice_plane_xz(double slice, double slab, sdr_slice_plane* out) {  // SlicePlane::xz, render.rs:78-89
    if (!out) {
        sdr_internal_set_error("null argument");
        return SDR_ERR_INVALID;
    }
    *out = sdr_slice_plane{0, 2, 1, 0, 0, 0, slice, slab};
    return SDR_OK;
}

int sdr_slice_plane_yz(double slice, double slab, sdr_slice_plane* out) {  // SlicePlane::yz, render.rs:92-103
    if (!out) {
        sdr_internal_set_error("null argument");
        return SDR_ERR_INVALID;
    }
    *out = sdr_slice_plane{1, 2, 0, 1, 0, 0, slice, slab};
    return SDR_OK;
}

// SlicePlane::projected_along_gravity (render.rs:113-136): look along the
// axis with the least gravity (first on ties), the larger remaining component
// vertical, flipped so +gravity points down; a silhouette with the amber pool.
int sdr_slice_plane_gravity(sdr_vec3 gravity, sdr_slice_plane* out) {
    if (!out) {
        sdr_internal_set_error("null argument");
        return SDR_ERR_INVALID;
    }
    const double g[3] = {gravity.x, gravity.y, gravity.z};
    const double ga[3] = {std::fabs(g[0]), std::fabs(g[1]), std::fabs(g[2])};
    int oax = 0;
    for (int a = 1; a < 3; ++a)
        if (ga[a] < ga[oax]) oax = a;
    int rem[2], k = 0;
    for (int a = 0; a < 3; ++a)
        if (a != oax) rem[k++] = a;
    const int vax = ga[rem[0]] >= ga[rem[1]] ? rem[0] : rem[1];
    const int hax = vax == rem[0] ? rem[1] : rem[0];
    *out = sdr_slice_plane{hax, vax, oax, g[vax] < 0.0 ? 1 : 0, 1, 1, 0.0, INFINITY};
    return SDR_OK;
}

// render_timeseries (render.rs:351-406): fill (blue), wall coverage (green)
// and the focal membrane load over its peak (red) on a 0..1 axis.
int sdr_render_timeseries(const sdr_frame_metrics* frames, size_t n, uint32_t width, uint32_t height, uint8_t* rgb,
                          size_t cap) {
    if ((n && !frames) || !rgb) {
        sdr_internal_set_error("null argument");
        return SDR_ERR_INVALID;
    }
    if (cap < (size_t)width * height * 3) {
        sdr_internal_set_error("image buffer too small: need " + std::to_string((size_t)width * height * 3) + " bytes");
        return SDR_ERR_BUFFER;
    }
    const uint8_t bg[3] = {250, 250, 252};
    for (size_t q = 0; q < (size_t)width * height; ++q) std::memcpy(rgb + 3 * q, bg, 3);
    const int64_t x0 = 8, x1 = (int64_t)width - 8, y0 = 8, y1 = (int64_t)height - 8;
    const uint8_t grid[3] = {220, 220, 226}, axis[3] = {120, 120, 130};
    for (int64_t g = 0; g <= 4; ++g) {
        const int64_t y = y1 - (y1 - y0) * g / 4;
        sdr_internal_draw_line(rgb, width, height, x0, y, x1, y, grid);
    }
    sdr_internal_draw_line(rgb, width, height, x0, y0, x0, y1, axis);
    sdr_internal_draw_line(rgb, width, height, x0, y1, x1, y1, axis);
    if (n < 2) return SDR_OK;
    double peak = 0.0;
    for (size_t i = 0; i < n; ++i) peak = std::fmax(peak, frames[i].peak_wall_pressure_pa);
    peak = std::fmax(peak, 1e-9);
    const uint8_t cols[3][3] = {{40, 90, 220}, {30, 160, 60}, {210, 60, 50}};
    for (int s = 0; s < 3; ++s) {
        auto val = [&](const sdr_frame_metrics& m) {
            return s == 0 ? m.fill_fraction : (s == 1 ? m.wall_coverage : m.peak_wall_pressure_pa / peak);
        };
        auto map = [&](size_t i, double v, int64_t& px, int64_t& py) {
            const double fx = (double)x0 + (double)(x1 - x0) * (double)i / (double)(n - 1);
            const double c = v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
            const double fy = (double)y1 - (double)(y1 - y0) * c;
            px = as_i64(fx);
            py = as_i64(fy);
        };
        for (size_t i = 1; i < n; ++i) {
            int64_t xa, ya, xb, yb;
            map(i - 1, val(frames[i - 1]), xa, ya);
            map(i, val(frames[i]), xb, yb);
            sdr_internal_draw_line(rgb, width, height, xa, ya, xb, yb, cols[s]);
        }
    }
    return SDR_OK;
}

// save_png (render.rs:409-414): 8-bit RGB, no interlace, rows unfiltered,
// zlib-deflated image data.
int sdr_write_png(const char* path, const uint8_t* rgb, uint32_t w, uint32_t h) {
    if (!path || !rgb || !w || !h) {
        sdr_internal_set_error("null argument or empty image");
        return SDR_ERR_INVALID;
    }
    std::vector<uint8_t> raw;
    raw.reserve((size_t)h * (3 * (size_t)w + 1));
    for (uint32_t y = 0; y < h; ++y) {
        raw.push_back(0);  // filter: none
        raw.insert(raw.end(), rgb + 3 * (size_t)y * w, rgb + 3 * ((size_t)y + 1) * w);
    }
    uLongf zn = compressBound((uLong)raw.size());
    std::vector<uint8_t> z(zn);
    if (compress2(z.data(), &zn, raw.data(), (uLong)raw.size(), 6) != Z_OK) {
        sdr_internal_set_error("deflate failed");
        return SDR_ERR_IO;
    }
    std::vector<uint8_t> o = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    std::vector<uint8_t> ihdr;
    be32(ihdr, w);
    be32(ihdr, h);
    const uint8_t rest[5] = {8, 2, 0, 0, 0};  // depth 8, RGB, deflate, adaptive filtering, no interlace
    ihdr.insert(ihdr.end(), rest, rest + 5);
    png_chunk(o, "IHDR", ihdr.data(), ihdr.size());
    png_chunk(o, "IDAT", z.data(), zn);
    png_chunk(o, "IEND", nullptr, 0);
    std::FILE* f = std::fopen(path, "wb");
    if (!f) {
        sdr_internal_set_error(std::string("creating ") + path + ": " + std::strerror(errno));
        return SDR_ERR_IO;
    }
    bool good = std::fwrite(o.data(), 1, o.size(), f) == o.size();
    good = (std::fclose(f) == 0) && good;
    if (!good) {
        sdr_internal_set_error(std::string("writing ") + path + ": " + std::strerror(errno));
        return SDR_ERR_IO;
    }
    return SDR_OK;
}

}  // extern "C"
