// Frame output (src/output.rs:23-122): particle positions as an ASCII
// legacy-VTK point cloud or as raw little-endian f32 XYZ triples, and the
// zero-padded frame file names.
//
// Numbers in the VTK text follow Rust's `{}` for f64 (the reference writes
// f64 positions): the shortest digits that read back to the same value, in
// fixed notation, no exponent ("0", "-0", "0.1", "0.0000001"). The device
// stores f32 positions; they are widened to f64 before formatting, which is
// what the reference would print for those values.
#include <cerrno>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "sdr_gpu.h"

void sdr_internal_set_error(const std::string& msg);

namespace {

size_t fmt_f64(char* out, double v) {
    if (std::isnan(v)) return (size_t)std::snprintf(out, 8, "NaN");
    if (std::isinf(v)) return (size_t)std::snprintf(out, 8, v < 0 ? "-inf" : "inf");
    auto r = std::to_chars(out, out + 400, v, std::chars_format::fixed);
    return (size_t)(r.ptr - out);
}

class Out {
   public:
    explicit Out(std::FILE* f) : f_(f) { buf_.reserve(1 << 20); }
    void put(const char* s, size_t n) {
        buf_.append(s, n);
        if (buf_.size() >= (1 << 20)) flush();
    }
    void put(const std::string& s) { put(s.data(), s.size()); }
    bool flush() {
        if (!buf_.empty() && std::fwrite(buf_.data(), 1, buf_.size(), f_) != buf_.size()) ok_ = false;
        buf_.clear();
        return ok_;
    }
    bool ok() const { return ok_; }

   private:
    std::FILE* f_;
    std::string buf_;
    bool ok_ = true;
};

}  // namespace

// Positions: n points, the i-th at xyz[i * stride + 0..2] (stride 3 for packed
// triples, 4 for the device's float4 layout). Returns SDR_OK or an error code
// with the message in `err`.
int sdr_internal_write_points(const char* path, int32_t format, const float* xyz, size_t stride, size_t n,
                              std::string& err) {
    if (format != SDR_FORMAT_VTK && format != SDR_FORMAT_XYZ) {
        err = "unknown output format " + std::to_string(format);
        return SDR_ERR_INVALID;
    }
    std::FILE* f = std::fopen(path, "wb");
    if (!f) {
        err = std::string("creating ") + path + ": " + std::strerror(errno);
        return SDR_ERR_IO;
    }
    Out o(f);
    if (format == SDR_FORMAT_VTK) {  // write_points_vtk, output.rs:23-48
        o.put("# vtk DataFile Version 4.2\nsdr irrigation particles\nASCII\nDATASET UNSTRUCTURED_GRID\n");
        o.put("POINTS " + std::to_string(n) + " double\n");
        char line[1300];
        for (size_t i = 0; i < n; ++i) {
            const float* p = xyz + i * stride;
            size_t k = fmt_f64(line, (double)p[0]);
            line[k++] = ' ';
            k += fmt_f64(line + k, (double)p[1]);
            line[k++] = ' ';
            k += fmt_f64(line + k, (double)p[2]);
            line[k++] = '\n';
            o.put(line, k);
        }
        o.put("CELLS " + std::to_string(n) + " " + std::to_string(n * 2) + "\n");
        for (size_t i = 0; i < n; ++i) o.put("1 " + std::to_string(i) + "\n");
        o.put("CELL_TYPES " + std::to_string(n) + "\n");
        for (size_t i = 0; i < n; ++i) o.put("1\n", 2);
    } else {  // write_points_xyz, output.rs:98-110: little-endian f32 triples, no header
        for (size_t i = 0; i < n; ++i) o.put(reinterpret_cast<const char*>(xyz + i * stride), 12);
    }
    bool good = o.flush();
    good = (std::fclose(f) == 0) && good;
    if (!good) {
        err = std::string("writing ") + path + ": " + std::strerror(errno);
        return SDR_ERR_IO;
    }
    return SDR_OK;
}

std::string sdr_internal_frame_path(const char* dir, const char* prefix, uint64_t frame, int32_t format) {
    char num[32];
    std::snprintf(num, sizeof num, "%06llu", (unsigned long long)frame);
    std::string d(dir ? dir : "");
    if (!d.empty() && d.back() != '/') d += '/';
    return d + (prefix ? prefix : "") + "_" + num + (format == SDR_FORMAT_XYZ ? ".xyz" : ".vtk");
}

extern "C" {

int sdr_write_points(const char* path, int32_t format, const float* xyz, size_t n) {
    if (!path || (n && !xyz)) {
        sdr_internal_set_error("null argument");
        return SDR_ERR_INVALID;
    }
    std::string err;
    int rc = sdr_internal_write_points(path, format, xyz, 3, n, err);
    if (rc != SDR_OK) sdr_internal_set_error(err);
    return rc;
}

int sdr_frame_path(const char* dir, const char* prefix, uint64_t frame, int32_t format, char* out, size_t cap) {
    if (!dir || !prefix || !out) {
        sdr_internal_set_error("null argument");
        return SDR_ERR_INVALID;
    }
    std::string p = sdr_internal_frame_path(dir, prefix, frame, format);
    if (p.size() + 1 > cap) {
        sdr_internal_set_error("buffer too small: need " + std::to_string(p.size() + 1) + " bytes");
        return SDR_ERR_BUFFER;
    }
    std::memcpy(out, p.c_str(), p.size() + 1);
    return SDR_OK;
}

}  // extern "C"
