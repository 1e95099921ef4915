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
#include <cstdlib>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "sdr_gpu.h"

void sdr_internal_set_error(const std::string& msg);

namespace {

// Shortest round-trip decimal digits of a finite a > 0: a = digits x 10^k.
int shortest_digits(double a, char* dig, int& k) {
    char sci[64];
    auto r = std::to_chars(sci, sci + sizeof sci - 1, a, std::chars_format::scientific);  // d.ddde+xx
    *r.ptr = '\0';
    int n = 0;
    const char* q = sci;
    for (; *q && *q != 'e'; ++q)
        if (*q != '.') dig[n++] = *q;
    k = std::atoi(q + 1) - (n - 1);
    return n;
}

// Rust's `{}` for f64: the shortest round-trip digits in plain notation, never
// an exponent, no fractional part for integral values ("0", "-0", "0.1",
// "0.0000001", "18446744073709552000").
size_t fmt_f64(char* out, double v) {
    if (std::isnan(v)) return (size_t)std::snprintf(out, 8, "NaN");
    if (std::isinf(v)) return (size_t)std::snprintf(out, 8, v < 0 ? "-inf" : "inf");
    size_t o = 0;
    if (std::signbit(v)) out[o++] = '-';
    const double a = std::fabs(v);
    if (a == 0.0) {
        out[o++] = '0';
        return o;
    }
    char dig[32];
    int k = 0;
    const int n = shortest_digits(a, dig, k);
    if (k >= 0) {
        std::memcpy(out + o, dig, n);
        o += n;
        for (int z = 0; z < k; ++z) out[o++] = '0';
    } else if (-k < n) {
        std::memcpy(out + o, dig, n + k);
        o += n + k;
        out[o++] = '.';
        std::memcpy(out + o, dig + n + k, -k);
        o += -k;
    } else {
        out[o++] = '0';
        out[o++] = '.';
        for (int z = 0; z < -k - n; ++z) out[o++] = '0';
        std::memcpy(out + o, dig, n);
        o += n;
    }
    return o;
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

// ---------------------------------------------------------------- metrics files
// serde_json (1.0.150 in the reference's lock file; floats through zmij
// 1.0.21, integers through itoa) writes an f64 as its shortest round-trip
// digits: in plain notation with at least one fractional digit when
// 1e-5 <= |v| < 1e16 ("0.0", "12.5", "1000.0", "0.00001"), otherwise as
// d[.ddd]e[-]x ("1e-6", "1.5e16"); non-finite values become null.
// to_string_pretty indents by two spaces and puts one member per line.
namespace {

size_t fmt_json_f64(char* out, double v) {
    if (!std::isfinite(v)) return (size_t)std::snprintf(out, 8, "null");
    size_t o = 0;
    if (std::signbit(v)) out[o++] = '-';
    const double a = std::fabs(v);
    if (a == 0.0) {
        std::memcpy(out + o, "0.0", 3);
        return o + 3;
    }
    char dig[32];
    int k = 0;                                   // value = digits x 10^k
    const int n = shortest_digits(a, dig, k);
    const int kk = n + k;                        // 10^(kk-1) <= value < 10^kk
    if (k >= 0 && kk <= 16) {        // 1234e7 -> 12340000000.0
        std::memcpy(out + o, dig, n);
        o += n;
        for (int z = n; z < kk; ++z) out[o++] = '0';
        out[o++] = '.';
        out[o++] = '0';
    } else if (kk > 0 && kk <= 16) {  // 1234e-2 -> 12.34
        std::memcpy(out + o, dig, kk);
        o += kk;
        out[o++] = '.';
        std::memcpy(out + o, dig + kk, n - kk);
        o += n - kk;
    } else if (kk > -5 && kk <= 0) {  // 1234e-6 -> 0.001234
        out[o++] = '0';
        out[o++] = '.';
        for (int z = 0; z < -kk; ++z) out[o++] = '0';
        std::memcpy(out + o, dig, n);
        o += n;
    } else {  // 1e30, 1.234e33, 1e-7
        out[o++] = dig[0];
        if (n > 1) {
            out[o++] = '.';
            std::memcpy(out + o, dig + 1, n - 1);
            o += n - 1;
        }
        o += (size_t)std::snprintf(out + o, 16, "e%d", kk - 1);
    }
    return o;
}

struct Field {
    const char* name;
    bool integer;
    double f;
    uint64_t u;
};

void frame_fields(const sdr_frame_metrics& m, Field* f) {  // FrameMetrics, metrics.rs:27-66 (field order)
    int i = 0;
    f[i++] = {"frame", true, 0, m.frame};
    f[i++] = {"time_s", false, m.time_s, 0};
    f[i++] = {"particles", true, 0, m.particles};
    f[i++] = {"fluid_volume_ml", false, m.fluid_volume_ml, 0};
    f[i++] = {"drained_volume_ml", false, m.drained_volume_ml, 0};
    f[i++] = {"fill_fraction", false, m.fill_fraction, 0};
    f[i++] = {"wall_coverage", false, m.wall_coverage, 0};
    f[i++] = {"mean_pressure_pa", false, m.mean_pressure_pa, 0};
    f[i++] = {"max_pressure_pa", false, m.max_pressure_pa, 0};
    f[i++] = {"max_pressure_mmhg", false, m.max_pressure_mmhg, 0};
    f[i++] = {"wall_pressure_pa", false, m.wall_pressure_pa, 0};
    f[i++] = {"peak_wall_pressure_pa", false, m.peak_wall_pressure_pa, 0};
    f[i++] = {"peak_wall_pressure_mmhg", false, m.peak_wall_pressure_mmhg, 0};
    f[i++] = {"membrane_artifacts", true, 0, m.membrane_artifacts};
    f[i++] = {"max_speed_m_s", false, m.max_speed_m_s, 0};
    f[i++] = {"kinetic_energy", false, m.kinetic_energy, 0};
    f[i++] = {"pcg_iters", true, 0, m.pcg_iters};
}
constexpr int kFrameFields = 17;

void summary_fields(const sdr_summary& s, Field* f) {  // Summary, metrics.rs:69-97 (field order)
    int i = 0;
    f[i++] = {"frames", true, 0, s.frames};
    f[i++] = {"final_time_s", false, s.final_time_s, 0};
    f[i++] = {"peak_fill_fraction", false, s.peak_fill_fraction, 0};
    f[i++] = {"final_fill_fraction", false, s.final_fill_fraction, 0};
    f[i++] = {"peak_wall_coverage", false, s.peak_wall_coverage, 0};
    f[i++] = {"final_wall_coverage", false, s.final_wall_coverage, 0};
    f[i++] = {"peak_membrane_pressure_pa", false, s.peak_membrane_pressure_pa, 0};
    f[i++] = {"peak_membrane_pressure_mmhg", false, s.peak_membrane_pressure_mmhg, 0};
    f[i++] = {"mean_membrane_pressure_pa", false, s.mean_membrane_pressure_pa, 0};
    f[i++] = {"mean_membrane_pressure_mmhg", false, s.mean_membrane_pressure_mmhg, 0};
    f[i++] = {"peak_pressure_pa", false, s.peak_pressure_pa, 0};
    f[i++] = {"peak_pressure_mmhg", false, s.peak_pressure_mmhg, 0};
    f[i++] = {"membrane_artifacts_total", true, 0, s.membrane_artifacts_total};
    f[i++] = {"total_drained_ml", false, s.total_drained_ml, 0};
    f[i++] = {"injected_ml", false, s.injected_ml, 0};
    f[i++] = {"mass_balance", false, s.mass_balance, 0};
}
constexpr int kSummaryFields = 16;

// One pretty-printed JSON object at the given indent (no trailing newline).
void json_object(std::string& t, const Field* f, int nf, const char* ind) {
    char num[400];
    t += "{\n";
    for (int i = 0; i < nf; ++i) {
        t += ind;
        t += "  \"";
        t += f[i].name;
        t += "\": ";
        if (f[i].integer) t += std::to_string(f[i].u);
        else t.append(num, fmt_json_f64(num, f[i].f));
        if (i + 1 < nf) t += ",";
        t += "\n";
    }
    t += ind;
    t += "}";
}

int write_text(const char* path, const std::string& t, std::string& err) {
    std::FILE* fp = std::fopen(path, "wb");
    if (!fp) {
        err = std::string("creating ") + path + ": " + std::strerror(errno);
        return SDR_ERR_IO;
    }
    bool good = std::fwrite(t.data(), 1, t.size(), fp) == t.size();
    good = (std::fclose(fp) == 0) && good;
    if (!good) {
        err = std::string("writing ") + path + ": " + std::strerror(errno);
        return SDR_ERR_IO;
    }
    return SDR_OK;
}

}  // namespace

// MetricsCollector::write_json (metrics.rs:385-391): the frames as a pretty JSON array.
std::string sdr_internal_frames_json(const sdr_frame_metrics* frames, size_t n) {
    if (n == 0) return "[]";
    std::string t = "[\n";
    Field f[kFrameFields];
    for (size_t i = 0; i < n; ++i) {
        frame_fields(frames[i], f);
        t += "  ";
        json_object(t, f, kFrameFields, "  ");
        t += i + 1 < n ? ",\n" : "\n";
    }
    t += "]";
    return t;
}

// MetricsCollector::write_csv (metrics.rs:394-431): header, then one row per
// frame with Rust's `{}` for every value.
std::string sdr_internal_frames_csv(const sdr_frame_metrics* frames, size_t n) {
    std::string t =
        "frame,time_s,particles,fluid_volume_ml,drained_volume_ml,fill_fraction,wall_coverage,"
        "mean_pressure_pa,max_pressure_pa,max_pressure_mmhg,"
        "wall_pressure_pa,peak_wall_pressure_pa,peak_wall_pressure_mmhg,membrane_artifacts,"
        "max_speed_m_s,kinetic_energy,pcg_iters\n";
    Field f[kFrameFields];
    char num[400];
    for (size_t i = 0; i < n; ++i) {
        frame_fields(frames[i], f);
        for (int j = 0; j < kFrameFields; ++j) {
            if (j) t += ",";
            if (f[j].integer) t += std::to_string(f[j].u);
            else t.append(num, fmt_f64(num, f[j].f));
        }
        t += "\n";
    }
    return t;
}

int sdr_internal_write_text(const char* path, const std::string& t, std::string& err) {
    return write_text(path, t, err);
}

extern "C" {

int sdr_frames_write_json(const sdr_frame_metrics* frames, size_t n, const char* path) {
    if (!path || (n && !frames)) {
        sdr_internal_set_error("null argument");
        return SDR_ERR_INVALID;
    }
    std::string err;
    int rc = write_text(path, sdr_internal_frames_json(frames, n), err);
    if (rc != SDR_OK) sdr_internal_set_error(err);
    return rc;
}

int sdr_frames_write_csv(const sdr_frame_metrics* frames, size_t n, const char* path) {
    if (!path || (n && !frames)) {
        sdr_internal_set_error("null argument");
        return SDR_ERR_INVALID;
    }
    std::string err;
    int rc = write_text(path, sdr_internal_frames_csv(frames, n), err);
    if (rc != SDR_OK) sdr_internal_set_error(err);
    return rc;
}

int sdr_summary_write_json(const sdr_summary* summary, const char* path) {
    if (!path || !summary) {
        sdr_internal_set_error("null argument");
        return SDR_ERR_INVALID;
    }
    Field f[kSummaryFields];
    summary_fields(*summary, f);
    std::string t;
    json_object(t, f, kSummaryFields, "");
    std::string err;
    int rc = write_text(path, t, err);
    if (rc != SDR_OK) sdr_internal_set_error(err);
    return rc;
}

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
