// sdr oracle — CPU restatement of uselessgoddess/sdr's FLIP/PIC substep, in f64.
//
// TEST INFRASTRUCTURE ONLY: this file is the checker for the CUDA path, never
// part of it. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
// leg load the library built from it.
//
// Every function follows the reference statement by statement, in the same
// f64 operation order (no FMA contraction: build with -ffp-contract=off), and
// cites the file:line it restates (paths relative to the reference project).
// The reference's rayon-parallel parts (apply_a, dot, axpys, inf_norm, SDF
// build) run on std::threads with the same deterministic reduction order, so
// results do not depend on the thread count.
#include "sdr_oracle.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <set>
#include <thread>
#include <condition_variable>
#include <memory>
#include <mutex>
#include <vector>

namespace {

// ---------------------------------------------------------------- threading
int g_threads = 0;  // 0 = hardware concurrency

int nthreads() {
    if (g_threads > 0) return g_threads;
    unsigned h = std::thread::hardware_concurrency();
    return h ? (int)h : 1;
}

// A persistent worker pool (like rayon's global pool): parallel_for splits
// [0, n) into one contiguous range per worker; the caller runs range 0.
// Workers spin briefly on a generation counter before sleeping, which keeps
// the per-call hand-off in the microsecond range like rayon's.
class Pool {
  public:
    explicit Pool(int n) : n_(n) {
        for (int w = 1; w < n_; ++w) ws_.emplace_back([this, w] { loop(w); });
    }
    ~Pool() {
        {
            std::lock_guard<std::mutex> g(m_);
            stop_ = true;
            gen_.fetch_add(1);
        }
        cv_.notify_all();
        for (auto& t : ws_) t.join();
    }
    int size() const { return n_; }
    void run(size_t n, const std::function<void(size_t, size_t)>& body) {
        body_ = &body;
        len_ = n;
        pending_.store(n_ - 1);
        {
            std::lock_guard<std::mutex> g(m_);
            gen_.fetch_add(1);
        }
        cv_.notify_all();
        range(0, n, body);
        while (pending_.load() != 0) std::this_thread::yield();
        body_ = nullptr;
    }

  private:
    void range(int w, size_t n, const std::function<void(size_t, size_t)>& body) {
        size_t per = (n + n_ - 1) / n_;
        size_t a = (size_t)w * per, b = std::min(n, a + per);
        if (a < b) body(a, b);
    }
    void loop(int w) {
        uint64_t seen = 0;
        for (;;) {
            auto t0 = std::chrono::steady_clock::now();
            while (gen_.load() == seen &&
                   std::chrono::steady_clock::now() - t0 < std::chrono::microseconds(200)) {
            }
            if (gen_.load() == seen) {
                std::unique_lock<std::mutex> g(m_);
                cv_.wait(g, [&] { return gen_.load() != seen; });
            }
            seen = gen_.load();
            if (stop_) return;
            range(w, len_, *body_);
            pending_.fetch_sub(1);
        }
    }
    int n_;
    std::vector<std::thread> ws_;
    std::mutex m_;
    std::condition_variable cv_;
    std::atomic<uint64_t> gen_{0};
    std::atomic<int> pending_{0};
    bool stop_ = false;
    size_t len_ = 0;
    const std::function<void(size_t, size_t)>* body_ = nullptr;
};

std::unique_ptr<Pool> g_pool;
std::mutex g_pool_m;

// `work` is the element count behind the n items (e.g. cells per z-slab x
// slabs); small loops stay serial, where a hand-off would cost more than it saves.
void parallel_for(size_t n, const std::function<void(size_t, size_t)>& body, size_t work = 0) {
    int t = nthreads();
    if (work == 0) work = n;
    if (t <= 1 || n < 2 || work < 32768) {
        body(0, n);
        return;
    }
    std::lock_guard<std::mutex> g(g_pool_m);
    if (!g_pool || g_pool->size() != t) g_pool.reset(new Pool(t));
    g_pool->run(n, body);
}

// ---------------------------------------------------------------- math.rs
struct V3 {
    double x, y, z;
};
inline V3 v3(double x, double y, double z) { return V3{x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator*(V3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
inline V3 operator/(V3 a, double s) { return v3(a.x / s, a.y / s, a.z / s); }
inline V3& operator+=(V3& a, V3 b) { a = a + b; return a; }
inline V3& operator-=(V3& a, V3 b) { a = a - b; return a; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }  // math.rs:42
inline V3 cross(V3 a, V3 b) {                                                 // math.rs:47
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline double length_sq(V3 a) { return dot(a, a); }
inline double length(V3 a) { return std::sqrt(length_sq(a)); }
// Rust f64::max/min ignore a NaN operand, like fmax/fmin.
inline double fmax_(double a, double b) { return std::fmax(a, b); }
inline double fmin_(double a, double b) { return std::fmin(a, b); }
inline V3 normalize_or_zero(V3 a) {  // math.rs:73-80
    double len = length(a);
    if (len > 1e-12) return a / len;
    return v3(0, 0, 0);
}
inline V3 vmin(V3 a, V3 b) { return v3(fmin_(a.x, b.x), fmin_(a.y, b.y), fmin_(a.z, b.z)); }
inline V3 vmax(V3 a, V3 b) { return v3(fmax_(a.x, b.x), fmax_(a.y, b.y), fmax_(a.z, b.z)); }
inline double min_component(V3 a) { return fmin_(fmin_(a.x, a.y), a.z); }
inline V3 from(const double* p) { return v3(p[0], p[1], p[2]); }
inline void to(V3 a, double* p) { p[0] = a.x; p[1] = a.y; p[2] = a.z; }
inline double clampd(double x, double lo, double hi) {  // Rust f64::clamp
    if (x < lo) return lo;
    if (x > hi) return hi;
    return x;
}

struct Aabb {  // math.rs:198-257
    V3 min, max;
    static Aabb empty() {
        double inf = std::numeric_limits<double>::infinity();
        return Aabb{v3(inf, inf, inf), v3(-inf, -inf, -inf)};
    }
    void expand(V3 p) { min = vmin(min, p); max = vmax(max, p); }
    V3 size() const { return max - min; }
    Aabb padded(double m) const { return Aabb{min - v3(m, m, m), max + v3(m, m, m)}; }
    bool contains(V3 p) const {
        return p.x >= min.x && p.x <= max.x && p.y >= min.y && p.y <= max.y && p.z >= min.z &&
               p.z <= max.z;
    }
};

// ---------------------------------------------------------------- grid.rs
struct Dims {
    size_t nx, ny, nz;
};

inline void clamp_base(double g, size_t n, size_t& i, double& f) {  // grid.rs:25-34
    if (g <= 0.0) {
        i = 0;
        f = 0.0;
    } else if (g >= (double)(n - 1)) {
        i = n - 2;
        f = 1.0;
    } else {
        double fl = std::floor(g);
        i = (size_t)fl;
        f = g - fl;
    }
}

double trilinear_sample(const double* arr, Dims d, double gx, double gy, double gz) {  // grid.rs:18-47
    size_t i, j, k;
    double fx, fy, fz;
    clamp_base(gx, d.nx, i, fx);
    clamp_base(gy, d.ny, j, fy);
    clamp_base(gz, d.nz, k, fz);
    auto at = [&](size_t a, size_t b, size_t c) { return arr[(c * d.ny + b) * d.nx + a]; };
    double c00 = at(i, j, k) * (1.0 - fx) + at(i + 1, j, k) * fx;
    double c10 = at(i, j + 1, k) * (1.0 - fx) + at(i + 1, j + 1, k) * fx;
    double c01 = at(i, j, k + 1) * (1.0 - fx) + at(i + 1, j, k + 1) * fx;
    double c11 = at(i, j + 1, k + 1) * (1.0 - fx) + at(i + 1, j + 1, k + 1) * fx;
    double c0 = c00 * (1.0 - fy) + c10 * fy;
    double c1 = c01 * (1.0 - fy) + c11 * fy;
    return c0 * (1.0 - fz) + c1 * fz;
}

void trilinear_scatter(double* arr, double* wsum, Dims d, double gx, double gy, double gz,
                       double val) {  // grid.rs:52-88
    size_t i, j, k;
    double fx, fy, fz;
    clamp_base(gx, d.nx, i, fx);
    clamp_base(gy, d.ny, j, fy);
    clamp_base(gz, d.nz, k, fz);
    double wx[2] = {1.0 - fx, fx}, wy[2] = {1.0 - fy, fy}, wz[2] = {1.0 - fz, fz};
    for (int dk = 0; dk < 2; ++dk)
        for (int dj = 0; dj < 2; ++dj)
            for (int di = 0; di < 2; ++di) {
                double w = wx[di] * wy[dj] * wz[dk];
                size_t idx = ((k + dk) * d.ny + (j + dj)) * d.nx + (i + di);
                arr[idx] += w * val;
                wsum[idx] += w;
            }
}

struct MacGrid {  // grid.rs:92-206
    size_t nx, ny, nz;
    double dx;
    V3 origin;
    std::vector<double> u, v, w;
    Dims ud() const { return {nx + 1, ny, nz}; }
    Dims vd() const { return {nx, ny + 1, nz}; }
    Dims wd() const { return {nx, ny, nz + 1}; }
    size_t u_idx(size_t i, size_t j, size_t k) const { return (k * ny + j) * (nx + 1) + i; }
    size_t v_idx(size_t i, size_t j, size_t k) const { return (k * (ny + 1) + j) * nx + i; }
    size_t w_idx(size_t i, size_t j, size_t k) const { return (k * ny + j) * nx + i; }
    V3 cell_center(size_t i, size_t j, size_t k) const {
        return origin + v3(((double)i + 0.5) * dx, ((double)j + 0.5) * dx, ((double)k + 0.5) * dx);
    }
    void u_coords(V3 p, double& gx, double& gy, double& gz) const {
        V3 l = (p - origin) / dx;
        gx = l.x; gy = l.y - 0.5; gz = l.z - 0.5;
    }
    void v_coords(V3 p, double& gx, double& gy, double& gz) const {
        V3 l = (p - origin) / dx;
        gx = l.x - 0.5; gy = l.y; gz = l.z - 0.5;
    }
    void w_coords(V3 p, double& gx, double& gy, double& gz) const {
        V3 l = (p - origin) / dx;
        gx = l.x - 0.5; gy = l.y - 0.5; gz = l.z;
    }
    V3 velocity_at(V3 p) const {  // grid.rs:191
        double gx, gy, gz;
        u_coords(p, gx, gy, gz);
        double a = trilinear_sample(u.data(), ud(), gx, gy, gz);
        v_coords(p, gx, gy, gz);
        double b = trilinear_sample(v.data(), vd(), gx, gy, gz);
        w_coords(p, gx, gy, gz);
        double c = trilinear_sample(w.data(), wd(), gx, gy, gz);
        return v3(a, b, c);
    }
    double max_speed() const {  // grid.rs:202-206
        auto m = [](const std::vector<double>& a) {
            double r = 0.0;
            for (double x : a) r = fmax_(r, std::fabs(x));
            return r;
        };
        double mu = m(u), mv = m(v), mw = m(w);
        return std::sqrt(mu * mu + mv * mv + mw * mw);
    }
};

// ---------------------------------------------------------------- sdf.rs
struct Sdf {  // sdf.rs:23-34
    V3 origin;
    double dx;
    size_t nx, ny, nz;
    std::vector<double> data;
    size_t idx(size_t i, size_t j, size_t k) const { return (k * ny + j) * nx + i; }
    Aabb bounds() const {  // sdf.rs:119-129
        return Aabb{origin, origin + v3((double)(nx - 1) * dx, (double)(ny - 1) * dx,
                                        (double)(nz - 1) * dx)};
    }
    double sample(V3 p) const {  // sdf.rs:134-166
        V3 l = (p - origin) / dx;
        size_t i, j, k;
        double fx, fy, fz;
        clamp_base(l.x, nx, i, fx);
        clamp_base(l.y, ny, j, fy);
        clamp_base(l.z, nz, k, fz);
        double c000 = data[idx(i, j, k)], c100 = data[idx(i + 1, j, k)];
        double c010 = data[idx(i, j + 1, k)], c110 = data[idx(i + 1, j + 1, k)];
        double c001 = data[idx(i, j, k + 1)], c101 = data[idx(i + 1, j, k + 1)];
        double c011 = data[idx(i, j + 1, k + 1)], c111 = data[idx(i + 1, j + 1, k + 1)];
        double c00 = c000 * (1.0 - fx) + c100 * fx;
        double c10 = c010 * (1.0 - fx) + c110 * fx;
        double c01 = c001 * (1.0 - fx) + c101 * fx;
        double c11 = c011 * (1.0 - fx) + c111 * fx;
        double c0 = c00 * (1.0 - fy) + c10 * fy;
        double c1 = c01 * (1.0 - fy) + c11 * fy;
        return c0 * (1.0 - fz) + c1 * fz;
    }
    V3 gradient(V3 p) const {  // sdf.rs:170-176
        double h = dx;
        double gx = sample(p + v3(h, 0, 0)) - sample(p - v3(h, 0, 0));
        double gy = sample(p + v3(0, h, 0)) - sample(p - v3(0, h, 0));
        double gz = sample(p + v3(0, 0, h)) - sample(p - v3(0, 0, h));
        return v3(gx, gy, gz) / (2.0 * h);
    }
};

double point_triangle_distance_sq(V3 p, V3 a, V3 b, V3 c) {  // sdf.rs:209-254
    V3 ab = b - a, ac = c - a, ap = p - a;
    double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) return length_sq(ap);
    V3 bp = p - b;
    double d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0 && d4 <= d3) return length_sq(bp);
    double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
        double v = d1 / (d1 - d3);
        V3 closest = a + ab * v;
        return length_sq(p - closest);
    }
    V3 cp = p - c;
    double d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0 && d5 <= d6) return length_sq(cp);
    double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        double w = d2 / (d2 - d6);
        V3 closest = a + ac * w;
        return length_sq(p - closest);
    }
    double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
        double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        V3 closest = b + (c - b) * w;
        return length_sq(p - closest);
    }
    double denom = 1.0 / (va + vb + vc);
    double v = vb * denom, w = vc * denom;
    V3 closest = a + ab * v + ac * w;
    return length_sq(p - closest);
}

double solid_angle(V3 p, V3 a, V3 b, V3 c) {  // sdf.rs:259-272
    V3 av = a - p, bv = b - p, cv = c - p;
    double la = length(av), lb = length(bv), lc = length(cv);
    if (la < 1e-12 || lb < 1e-12 || lc < 1e-12) return 0.0;
    double num = dot(av, cross(bv, cv));
    double den = la * lb * lc + dot(av, bv) * lc + dot(bv, cv) * la + dot(cv, av) * lb;
    return 2.0 * std::atan2(num, den);
}

double signed_distance_to_mesh(V3 p, const double* tris, size_t ntri) {  // sdf.rs:187-205
    double min_d2 = std::numeric_limits<double>::infinity();
    double winding = 0.0;
    for (size_t t = 0; t < ntri; ++t) {
        V3 a = from(tris + 9 * t), b = from(tris + 9 * t + 3), c = from(tris + 9 * t + 6);
        double d2 = point_triangle_distance_sq(p, a, b, c);
        if (d2 < min_d2) min_d2 = d2;
        winding += solid_angle(p, a, b, c);
    }
    winding /= 4.0 * M_PI;
    double dist = std::sqrt(min_d2);
    return winding > 0.5 ? -dist : dist;
}

// ---------------------------------------------------------------- sinus.rs
struct Sinus {
    V3 semi_axes, center;
    double taper, bumpiness, sx, sz, socket_radius, socket_depth, model_dx;
    double socket_bottom_y() const { return center.y - semi_axes.y - socket_depth; }  // sinus.rs:77
    double socket_top_y() const { return center.y - 0.5 * semi_axes.y; }              // sinus.rs:83
    double implicit(V3 p) const {                                                     // sinus.rs:89-119
        V3 q = p - center;
        V3 a = semi_axes;
        double h = ((q.y / a.y) + 1.0) * 0.5;
        double scale = taper + (1.0 - taper) * clampd(h, 0.0, 1.5);
        double bump = bumpiness * (0.6 * std::sin(4.0 * q.x / a.x) * std::cos(3.0 * q.z / a.z) +
                                   0.4 * std::sin(5.0 * q.y / a.y + 1.3));
        double tx = q.x / (a.x * scale), ty = q.y / a.y, tz = q.z / (a.z * scale);
        double body = std::sqrt(tx * tx + ty * ty + tz * tz) - (1.0 + bump);
        body = body * min_component(a);
        double rx = p.x - sx, rz = p.z - sz;
        double radial = std::sqrt(rx * rx + rz * rz) - socket_radius;
        double ytop = socket_top_y(), ybot = socket_bottom_y();
        double axial = fmax_(p.y - ytop, ybot - p.y);
        double socket = fmax_(radial, axial);
        // smooth_min, sinus.rs:66-72
        double k = 0.0015;
        double hh = clampd(0.5 + 0.5 * (socket - body) / k, 0.0, 1.0);
        return (socket * (1.0 - hh) + body * hh) - k * hh * (1.0 - hh);
    }
    Aabb bounds() const {  // sinus.rs:122-138
        V3 a = semi_axes * (1.0 + bumpiness);
        Aabb bb{center - a, center + a};
        bb.expand(v3(sx + socket_radius, socket_bottom_y(), sz + socket_radius));
        bb.expand(v3(sx - socket_radius, socket_bottom_y(), sz - socket_radius));
        return bb.padded(2.0 * model_dx);
    }
};

Sinus to_sinus(const orc_sinus* s) {
    Sinus r;
    r.semi_axes = from(s->semi_axes);
    r.center = from(s->center);
    r.taper = s->taper;
    r.bumpiness = s->bumpiness;
    r.sx = s->socket_xz[0];
    r.sz = s->socket_xz[1];
    r.socket_radius = s->socket_radius;
    r.socket_depth = s->socket_depth;
    r.model_dx = s->model_dx;
    return r;
}

// ---------------------------------------------------------------- surface_nets.rs
const int CORNERS[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {1, 1, 0},
                           {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
const int EDGES[12][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {0, 2}, {1, 3},
                          {4, 6}, {5, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};

void emit_quad(const int64_t ring[4], V3 desired, const std::vector<V3>& verts,
               std::vector<uint32_t>& idx) {  // surface_nets.rs:199-221
    for (int q = 0; q < 4; ++q)
        if (ring[q] < 0) return;
    uint32_t a = ring[0], b = ring[1], c = ring[2], d = ring[3];
    V3 n = cross(verts[b] - verts[a], verts[c] - verts[a]);
    if (dot(n, desired) >= 0.0) {
        idx.insert(idx.end(), {a, b, c, a, c, d});
    } else {
        idx.insert(idx.end(), {a, c, b, a, d, c});
    }
}

// surface_nets.rs:48-195; returns vertices and triangle indices.
void surface_nets(V3 origin, double dx, size_t nx, size_t ny, size_t nz,
                  const std::function<double(V3)>& field, std::vector<V3>& verts,
                  std::vector<uint32_t>& idx) {
    std::vector<double> values(nx * ny * nz);
    parallel_for(nz, [&](size_t k0, size_t k1) {
        for (size_t k = k0; k < k1; ++k)
            for (size_t j = 0; j < ny; ++j)
                for (size_t i = 0; i < nx; ++i)
                    values[(k * ny + j) * nx + i] =
                        field(origin + v3((double)i * dx, (double)j * dx, (double)k * dx));
    }, nx * ny * nz);
    auto node = [&](size_t i, size_t j, size_t k) { return values[(k * ny + j) * nx + i]; };
    size_t cx = nx - 1, cy = ny - 1, cz = nz - 1;
    std::vector<int64_t> cell_vertex(cx * cy * cz, -1);
    auto cidx = [&](size_t i, size_t j, size_t k) { return (k * cy + j) * cx + i; };
    verts.clear();
    for (size_t k = 0; k < cz; ++k)
        for (size_t j = 0; j < cy; ++j)
            for (size_t i = 0; i < cx; ++i) {
                double vals[8];
                for (int c = 0; c < 8; ++c)
                    vals[c] = node(i + CORNERS[c][0], j + CORNERS[c][1], k + CORNERS[c][2]);
                V3 sum = v3(0, 0, 0);
                int n = 0;
                for (int e = 0; e < 12; ++e) {
                    int a = EDGES[e][0], b = EDGES[e][1];
                    double va = vals[a], vb = vals[b];
                    if ((va < 0.0) != (vb < 0.0)) {
                        double t = va / (va - vb);
                        V3 pa = v3(CORNERS[a][0], CORNERS[a][1], CORNERS[a][2]);
                        V3 pb = v3(CORNERS[b][0], CORNERS[b][1], CORNERS[b][2]);
                        sum += pa + (pb - pa) * t;
                        ++n;
                    }
                }
                if (n == 0) continue;
                V3 local = sum / (double)n;
                V3 world = origin + v3(((double)i + local.x) * dx, ((double)j + local.y) * dx,
                                       ((double)k + local.z) * dx);
                cell_vertex[cidx(i, j, k)] = (int64_t)verts.size();
                verts.push_back(world);
            }
    idx.clear();
    auto get = [&](size_t i, size_t j, size_t k) { return cell_vertex[cidx(i, j, k)]; };
    for (size_t k = 0; k < nz; ++k)
        for (size_t j = 0; j < ny; ++j)
            for (size_t i = 0; i < nx; ++i) {
                double v0 = node(i, j, k);
                if (i + 1 < nx && j >= 1 && k >= 1) {
                    double v1 = node(i + 1, j, k);
                    if ((v0 < 0.0) != (v1 < 0.0)) {
                        int64_t ring[4] = {get(i, j - 1, k - 1), get(i, j, k - 1), get(i, j, k),
                                           get(i, j - 1, k)};
                        emit_quad(ring, v0 < v1 ? v3(1, 0, 0) : v3(-1, 0, 0), verts, idx);
                    }
                }
                if (j + 1 < ny && i >= 1 && k >= 1) {
                    double v1 = node(i, j + 1, k);
                    if ((v0 < 0.0) != (v1 < 0.0)) {
                        int64_t ring[4] = {get(i - 1, j, k - 1), get(i, j, k - 1), get(i, j, k),
                                           get(i - 1, j, k)};
                        emit_quad(ring, v0 < v1 ? v3(0, 1, 0) : v3(0, -1, 0), verts, idx);
                    }
                }
                if (k + 1 < nz && i >= 1 && j >= 1) {
                    double v1 = node(i, j, k + 1);
                    if ((v0 < 0.0) != (v1 < 0.0)) {
                        int64_t ring[4] = {get(i - 1, j - 1, k), get(i, j - 1, k), get(i, j, k),
                                           get(i - 1, j, k)};
                        emit_quad(ring, v0 < v1 ? v3(0, 0, 1) : v3(0, 0, -1), verts, idx);
                    }
                }
            }
}

double signed_volume(const std::vector<V3>& verts, const std::vector<uint32_t>& idx) {  // mesh.rs:63-70
    double v = 0.0;
    for (size_t t = 0; t + 2 < idx.size(); t += 3) {
        V3 a = verts[idx[t]], b = verts[idx[t + 1]], c = verts[idx[t + 2]];
        v += dot(a, cross(b, c)) / 6.0;
    }
    return v;
}

void sinus_mesh(const Sinus& s, std::vector<V3>& verts, std::vector<uint32_t>& idx) {  // sinus.rs:141-150
    Aabb bb = s.bounds();
    V3 size = bb.size();
    size_t nx = (size_t)std::ceil(size.x / s.model_dx) + 1;
    size_t ny = (size_t)std::ceil(size.y / s.model_dx) + 1;
    size_t nz = (size_t)std::ceil(size.z / s.model_dx) + 1;
    surface_nets(bb.min, s.model_dx, nx, ny, nz, [&](V3 p) { return s.implicit(p); }, verts, idx);
}

// ---------------------------------------------------------------- pressure.rs
enum : uint8_t { SOLID = 0, FLUID = 1, AIR = 2 };

struct Laplacian {  // pressure.rs:62-77
    std::vector<double> diag, plus_x, plus_y, plus_z;
    size_t nx, ny, nz;
    size_t idx(size_t i, size_t j, size_t k) const { return (k * ny + j) * nx + i; }
};

double dot_det(const double* a, const double* b, size_t n) {  // pressure.rs:588-603
    const size_t CHUNK = 4096;
    size_t nch = (n + CHUNK - 1) / CHUNK;
    std::vector<double> partials(nch);
    parallel_for(nch, [&](size_t c0, size_t c1) {
        for (size_t c = c0; c < c1; ++c) {
            double acc = 0.0;
            size_t e = std::min(n, (c + 1) * CHUNK);
            for (size_t i = c * CHUNK; i < e; ++i) acc += a[i] * b[i];
            partials[c] = acc;
        }
    }, n);
    // Rust's f64 Sum folds from -0.0 (identical to +0.0 for any non-(-0.0) input).
    double s = -0.0;
    for (double p : partials) s += p;
    return s;
}

double inf_norm(const std::vector<double>& a) {  // pressure.rs:605-609
    int t = nthreads();
    std::vector<double> parts(std::max(t, 1), 0.0);
    size_t n = a.size();
    size_t per = (n + parts.size() - 1) / parts.size();
    parallel_for(parts.size(), [&](size_t w0, size_t w1) {
        for (size_t w = w0; w < w1; ++w) {
            double m = 0.0;
            size_t e = std::min(n, (w + 1) * per);
            for (size_t i = w * per; i < e; ++i) m = fmax_(m, std::fabs(a[i]));
            parts[w] = m;
        }
    }, n);
    double m = 0.0;
    for (double p : parts) m = fmax_(m, p);
    return m;
}

void apply_a(const Laplacian& a, const uint8_t* cells, const double* x, double* out) {  // pressure.rs:400-439
    size_t nx = a.nx, ny = a.ny, nz = a.nz;
    parallel_for(nz, [&](size_t k0, size_t k1) {
        for (size_t k = k0; k < k1; ++k)
            for (size_t j = 0; j < ny; ++j)
                for (size_t i = 0; i < nx; ++i) {
                    size_t c = (k * ny + j) * nx + i;
                    if (cells[c] != FLUID) {
                        out[c] = 0.0;
                        continue;
                    }
                    double v = a.diag[c] * x[c];
                    if (i + 1 < nx) v += a.plus_x[c] * x[a.idx(i + 1, j, k)];
                    if (i >= 1) v += a.plus_x[a.idx(i - 1, j, k)] * x[a.idx(i - 1, j, k)];
                    if (j + 1 < ny) v += a.plus_y[c] * x[a.idx(i, j + 1, k)];
                    if (j >= 1) v += a.plus_y[a.idx(i, j - 1, k)] * x[a.idx(i, j - 1, k)];
                    if (k + 1 < nz) v += a.plus_z[c] * x[a.idx(i, j, k + 1)];
                    if (k >= 1) v += a.plus_z[a.idx(i, j, k - 1)] * x[a.idx(i, j, k - 1)];
                    out[c] = v;
                }
    }, nx * ny * nz);
}

std::vector<double> build_mic0(const Laplacian& a, const uint8_t* cells) {  // pressure.rs:442-513
    const double TAU = 0.97, SIGMA = 0.25;
    size_t nx = a.nx, ny = a.ny, nz = a.nz;
    std::vector<double> precon(nx * ny * nz, 0.0);
    for (size_t k = 0; k < nz; ++k)
        for (size_t j = 0; j < ny; ++j)
            for (size_t i = 0; i < nx; ++i) {
                size_t c = (k * ny + j) * nx + i;
                if (cells[c] != FLUID) continue;
                double axi = 0, pxi = 0, ayj = 0, pyj = 0, azk = 0, pzk = 0;
                double axi_y = 0, axi_z = 0, ayj_x = 0, ayj_z = 0, azk_x = 0, azk_y = 0;
                if (i >= 1) {
                    size_t cm = a.idx(i - 1, j, k);
                    axi = a.plus_x[cm]; pxi = precon[cm];
                    axi_y = a.plus_y[cm]; axi_z = a.plus_z[cm];
                }
                if (j >= 1) {
                    size_t cm = a.idx(i, j - 1, k);
                    ayj = a.plus_y[cm]; pyj = precon[cm];
                    ayj_x = a.plus_x[cm]; ayj_z = a.plus_z[cm];
                }
                if (k >= 1) {
                    size_t cm = a.idx(i, j, k - 1);
                    azk = a.plus_z[cm]; pzk = precon[cm];
                    azk_x = a.plus_x[cm]; azk_y = a.plus_y[cm];
                }
                double term_x = axi * pxi, term_y = ayj * pyj, term_z = azk * pzk;
                double e = a.diag[c] - term_x * term_x - term_y * term_y - term_z * term_z -
                           TAU * (axi * (axi_y + axi_z) * pxi * pxi +
                                  ayj * (ayj_x + ayj_z) * pyj * pyj +
                                  azk * (azk_x + azk_y) * pzk * pzk);
                if (e < SIGMA * a.diag[c]) e = a.diag[c];
                precon[c] = e > 0.0 ? 1.0 / std::sqrt(e) : 0.0;
            }
    return precon;
}

void apply_mic0(const Laplacian& a, const std::vector<double>& precon, const uint8_t* cells,
                const double* r, double* z, std::vector<double>& q) {  // pressure.rs:517-570
    size_t nx = a.nx, ny = a.ny, nz = a.nz;
    std::fill(q.begin(), q.end(), 0.0);
    for (size_t k = 0; k < nz; ++k)
        for (size_t j = 0; j < ny; ++j)
            for (size_t i = 0; i < nx; ++i) {
                size_t c = (k * ny + j) * nx + i;
                if (cells[c] != FLUID) continue;
                double t = r[c];
                if (i >= 1) { size_t cm = a.idx(i - 1, j, k); t -= a.plus_x[cm] * precon[cm] * q[cm]; }
                if (j >= 1) { size_t cm = a.idx(i, j - 1, k); t -= a.plus_y[cm] * precon[cm] * q[cm]; }
                if (k >= 1) { size_t cm = a.idx(i, j, k - 1); t -= a.plus_z[cm] * precon[cm] * q[cm]; }
                q[c] = t * precon[c];
            }
    for (size_t k = nz; k-- > 0;)
        for (size_t j = ny; j-- > 0;)
            for (size_t i = nx; i-- > 0;) {
                size_t c = (k * ny + j) * nx + i;
                if (cells[c] != FLUID) { z[c] = 0.0; continue; }
                double t = q[c];
                if (i + 1 < nx) t -= a.plus_x[c] * precon[c] * z[a.idx(i + 1, j, k)];
                if (j + 1 < ny) t -= a.plus_y[c] * precon[c] * z[a.idx(i, j + 1, k)];
                if (k + 1 < nz) t -= a.plus_z[c] * precon[c] * z[a.idx(i, j, k + 1)];
                z[c] = t * precon[c];
            }
}

struct PcgResult {
    std::vector<double> pressure;
    size_t iters;
    double residual;
};

PcgResult pcg(const Laplacian& a, const uint8_t* cells, const std::vector<double>& b,
              size_t max_iters, double tol) {  // pressure.rs:341-397
    size_t n = b.size();
    std::vector<double> p(n, 0.0);
    double residual = inf_norm(b);
    if (residual <= tol) return {p, 0, residual};
    std::vector<double> precon = build_mic0(a, cells);
    std::vector<double> r = b, z(n, 0.0), q(n, 0.0);
    apply_mic0(a, precon, cells, r.data(), z.data(), q);
    std::vector<double> s = z;
    double sigma = dot_det(z.data(), r.data(), n);
    std::vector<double> as(n, 0.0);
    size_t iters = 0;
    for (size_t it = 0; it < max_iters; ++it) {
        iters = it + 1;
        apply_a(a, cells, s.data(), as.data());
        double denom = dot_det(s.data(), as.data(), n);
        if (std::fabs(denom) < 1e-30) break;
        double alpha = sigma / denom;
        parallel_for(n, [&](size_t i0, size_t i1) {
            for (size_t i = i0; i < i1; ++i) p[i] += alpha * s[i];
        });
        parallel_for(n, [&](size_t i0, size_t i1) {
            for (size_t i = i0; i < i1; ++i) r[i] -= alpha * as[i];
        });
        residual = inf_norm(r);
        if (residual <= tol) break;
        apply_mic0(a, precon, cells, r.data(), z.data(), q);
        double sigma_new = dot_det(z.data(), r.data(), n);
        double beta = sigma_new / sigma;
        parallel_for(n, [&](size_t i0, size_t i1) {
            for (size_t i = i0; i < i1; ++i) s[i] = z[i] + beta * s[i];
        });
        sigma = sigma_new;
    }
    return {p, iters, residual};
}

void enforce_solid_faces(MacGrid& g, const uint8_t* cells) {  // pressure.rs:243-281
    size_t nx = g.nx, ny = g.ny, nz = g.nz;
    auto solid = [&](int64_t i, int64_t j, int64_t k) {
        if (i < 0 || j < 0 || k < 0 || (size_t)i >= nx || (size_t)j >= ny || (size_t)k >= nz)
            return true;
        return cells[((size_t)k * ny + (size_t)j) * nx + (size_t)i] == SOLID;
    };
    for (size_t k = 0; k < nz; ++k)
        for (size_t j = 0; j < ny; ++j)
            for (size_t i = 0; i <= nx; ++i)
                if (solid((int64_t)i - 1, j, k) || solid(i, j, k)) g.u[g.u_idx(i, j, k)] = 0.0;
    for (size_t k = 0; k < nz; ++k)
        for (size_t j = 0; j <= ny; ++j)
            for (size_t i = 0; i < nx; ++i)
                if (solid(i, (int64_t)j - 1, k) || solid(i, j, k)) g.v[g.v_idx(i, j, k)] = 0.0;
    for (size_t k = 0; k <= nz; ++k)
        for (size_t j = 0; j < ny; ++j)
            for (size_t i = 0; i < nx; ++i)
                if (solid(i, j, (int64_t)k - 1) || solid(i, j, k)) g.w[g.w_idx(i, j, k)] = 0.0;
}

void apply_pressure_gradient(MacGrid& g, const uint8_t* cells, const double* p, double coef) {  // pressure.rs:285-332
    size_t nx = g.nx, ny = g.ny, nz = g.nz;
    auto at = [&](size_t i, size_t j, size_t k) { return cells[(k * ny + j) * nx + i]; };
    auto pr = [&](size_t i, size_t j, size_t k) { return p[(k * ny + j) * nx + i]; };
    for (size_t k = 0; k < nz; ++k)
        for (size_t j = 0; j < ny; ++j)
            for (size_t i = 1; i < nx; ++i) {
                uint8_t l = at(i - 1, j, k), r = at(i, j, k);
                if (l == SOLID || r == SOLID) continue;
                if (l == FLUID || r == FLUID) g.u[g.u_idx(i, j, k)] -= coef * (pr(i, j, k) - pr(i - 1, j, k));
            }
    for (size_t k = 0; k < nz; ++k)
        for (size_t j = 1; j < ny; ++j)
            for (size_t i = 0; i < nx; ++i) {
                uint8_t l = at(i, j - 1, k), r = at(i, j, k);
                if (l == SOLID || r == SOLID) continue;
                if (l == FLUID || r == FLUID) g.v[g.v_idx(i, j, k)] -= coef * (pr(i, j, k) - pr(i, j - 1, k));
            }
    for (size_t k = 1; k < nz; ++k)
        for (size_t j = 0; j < ny; ++j)
            for (size_t i = 0; i < nx; ++i) {
                uint8_t l = at(i, j, k - 1), r = at(i, j, k);
                if (l == SOLID || r == SOLID) continue;
                if (l == FLUID || r == FLUID) g.w[g.w_idx(i, j, k)] -= coef * (pr(i, j, k) - pr(i, j, k - 1));
            }
}

// pressure.rs:123-239
PcgResult project_with_source(MacGrid& g, const uint8_t* cells, double rho, double dt,
                              size_t max_iters, double tol, const double* source) {
    size_t nx = g.nx, ny = g.ny, nz = g.nz, n = nx * ny * nz;
    enforce_solid_faces(g, cells);
    double inv_scale = rho * g.dx / dt;
    std::vector<double> b(n, 0.0);
    for (size_t k = 0; k < nz; ++k)
        for (size_t j = 0; j < ny; ++j)
            for (size_t i = 0; i < nx; ++i) {
                size_t c = (k * ny + j) * nx + i;
                if (cells[c] != FLUID) continue;
                double div = (g.u[g.u_idx(i + 1, j, k)] - g.u[g.u_idx(i, j, k)]) +
                             (g.v[g.v_idx(i, j + 1, k)] - g.v[g.v_idx(i, j, k)]) +
                             (g.w[g.w_idx(i, j, k + 1)] - g.w[g.w_idx(i, j, k)]);
                double s = source ? source[c] : 0.0;
                b[c] = -inv_scale * (div - s);
            }
    Laplacian a;
    a.nx = nx; a.ny = ny; a.nz = nz;
    a.diag.assign(n, 0.0); a.plus_x.assign(n, 0.0); a.plus_y.assign(n, 0.0); a.plus_z.assign(n, 0.0);
    auto cell = [&](size_t i, size_t j, size_t k) { return cells[(k * ny + j) * nx + i]; };
    for (size_t k = 0; k < nz; ++k)
        for (size_t j = 0; j < ny; ++j)
            for (size_t i = 0; i < nx; ++i) {
                size_t c = (k * ny + j) * nx + i;
                if (cells[c] != FLUID) continue;
                double diag = 0.0;
                auto consider = [&](int64_t ni, int64_t nj, int64_t nk, double* plus) {
                    bool inside = ni >= 0 && nj >= 0 && nk >= 0 && (size_t)ni < nx &&
                                  (size_t)nj < ny && (size_t)nk < nz;
                    uint8_t kind = inside ? cell(ni, nj, nk) : SOLID;
                    if (kind == AIR) diag += 1.0;
                    else if (kind == FLUID) {
                        diag += 1.0;
                        if (plus) *plus = -1.0;
                    }
                };
                int64_t ii = i, jj = j, kk = k;
                consider(ii - 1, jj, kk, nullptr);
                consider(ii + 1, jj, kk, &a.plus_x[c]);
                consider(ii, jj - 1, kk, nullptr);
                consider(ii, jj + 1, kk, &a.plus_y[c]);
                consider(ii, jj, kk - 1, nullptr);
                consider(ii, jj, kk + 1, &a.plus_z[c]);
                a.diag[c] = diag;
            }
    PcgResult rep = pcg(a, cells, b, max_iters, tol);
    double coef = dt / (rho * g.dx);
    apply_pressure_gradient(g, cells, rep.pressure.data(), coef);
    return rep;
}

// ---------------------------------------------------------------- solver.rs
struct Rng {  // solver.rs:120-140
    uint64_t s;
    uint64_t next_u64() {
        uint64_t x = s;
        x ^= x << 13;
        x ^= x >> 7;
        x ^= x << 17;
        s = x;
        return x;
    }
    double unit() { return (double)(next_u64() >> 11) / (double)(1ULL << 53); }
};

V3 hash_jitter(uint64_t key) {  // solver.rs:916-930
    auto mix = [](uint64_t k) {
        uint64_t z = k + 0x9E3779B97F4A7C15ULL;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        return ((double)(z >> 11) / (double)(1ULL << 53) - 0.5) * 0.6;
    };
    return v3(mix(key * 3), mix(key * 3 + 1), mix(key * 3 + 2));
}

void orthonormal_basis(V3 n, V3& e1, V3& e2) {  // solver.rs:933-942
    V3 a = std::fabs(n.x) < 0.9 ? v3(1, 0, 0) : v3(0, 1, 0);
    e1 = normalize_or_zero(cross(n, a));
    e2 = normalize_or_zero(cross(n, e1));
}

struct Fluid {
    double density;
    V3 gravity;
    double flip_ratio;
    size_t ppc;
    double volume_stiffness;
    bool redistribute;
    double redist_cap_factor;
};

struct Needle {
    V3 tip, axis;
    double radius, flow_rate, inject_until;
    double jet_speed() const {  // solver.rs:107-114
        double area = M_PI * radius * radius;
        return area > 0.0 ? flow_rate / area : 0.0;
    }
};

const double VC_MAX_FRACTION = 0.25;  // solver.rs:31
const size_t REDIST_SWEEPS = 4;       // solver.rs:37

}  // namespace

struct orc_solver {  // solver.rs:143-180
    MacGrid grid;
    std::vector<V3> pos, vel;
    Sdf solid;
    Fluid fluid;
    Needle needle;
    bool has_outlet = false;
    Aabb outlet;
    size_t max_iters = 200;
    double tol = 1e-6;
    double time = 0.0;
    uint64_t steps = 0;
    uint64_t last_pcg_iters = 0;
    uint64_t last_substeps = 0;
    std::vector<double> pressure;
    uint64_t drained = 0;
    std::vector<uint8_t> cells;
    std::vector<uint8_t> cavity_mask;
    std::vector<double> saved_u, saved_v, saved_w;
    Rng rng{0x5deece66dULL | 1ULL};
    double emit_accum = 0.0;
    double phase_t[12] = {0};

    double particle_volume() const {  // solver.rs:225-228
        double cell = grid.dx * grid.dx * grid.dx;
        return cell / (double)std::max<size_t>(fluid.ppc, 1);
    }
    double fluid_volume() const { return (double)pos.size() * particle_volume(); }
    double drained_volume() const { return (double)drained * particle_volume(); }
    bool in_outlet(V3 p) const { return has_outlet && outlet.contains(p); }

    bool cell_of(V3 p, size_t& i, size_t& j, size_t& k) const {  // solver.rs:897-908
        V3 l = (p - grid.origin) / grid.dx;
        if (l.x < 0.0 || l.y < 0.0 || l.z < 0.0) return false;
        // `as usize` saturates; values are non-negative here.
        double mx = 1.8e19;
        i = l.x >= mx ? SIZE_MAX : (size_t)l.x;
        j = l.y >= mx ? SIZE_MAX : (size_t)l.y;
        k = l.z >= mx ? SIZE_MAX : (size_t)l.z;
        return i < grid.nx && j < grid.ny && k < grid.nz;
    }

    double cfl_dt() const {  // solver.rs:262-281
        double grid_speed = grid.max_speed();
        double jet = time < needle.inject_until ? needle.jet_speed() : 0.0;
        double g = std::sqrt(length(fluid.gravity) * grid.dx);
        double speed = fmax_(fmax_(fmax_(grid_speed, jet), g), 1e-6);
        return fmin_(grid.dx / speed, 0.01);
    }

    void step(double dt) {  // solver.rs:237-259
        const uint32_t MAX_SUBSTEPS = 512;
        double floor_ = dt / (double)MAX_SUBSTEPS;
        double remaining = dt;
        uint32_t taken = 0;
        while (remaining > 1e-12) {
            double sub = fmin_(fmax_(cfl_dt(), floor_), remaining);
            substep(sub);
            remaining -= sub;
            ++taken;
        }
        last_substeps = taken;
    }

    void substep(double dt) {  // solver.rs:284-310
        for (int ph = ORC_PHASE_EMIT; ph <= ORC_PHASE_CLOCK; ++ph) phase(ph, dt);
    }

    void phase(int ph, double dt) {
        auto t0 = std::chrono::steady_clock::now();
        switch (ph) {
            case ORC_PHASE_EMIT: emit(dt); break;
            case ORC_PHASE_CLASSIFY: classify(); break;
            case ORC_PHASE_P2G: p2g(); break;
            case ORC_PHASE_SAVE_GRID: saved_u = grid.u; saved_v = grid.v; saved_w = grid.w; break;
            case ORC_PHASE_ADD_FORCES: add_forces(dt); break;
            case ORC_PHASE_PROJECT: {
                std::vector<double> src = volume_source(dt);
                PcgResult rep = project_with_source(grid, cells.data(), fluid.density, dt,
                                                    max_iters, tol, src.data());
                last_pcg_iters = rep.iters;
                pressure = std::move(rep.pressure);
                break;
            }
            case ORC_PHASE_EXTRAPOLATE: extrapolate_velocities(); break;
            case ORC_PHASE_G2P: g2p(); break;
            case ORC_PHASE_ADVECT: advect(dt); break;
            case ORC_PHASE_BOUNDS: enforce_particle_bounds(); break;
            case ORC_PHASE_REDISTRIBUTE:
                if (fluid.redistribute) redistribute();
                break;
            case ORC_PHASE_CLOCK: time += dt; steps += 1; break;
            default: break;
        }
        phase_t[ph] += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }

    void emit(double dt) {  // solver.rs:313-339
        double pv = particle_volume();
        if (pv <= 0.0 || needle.flow_rate <= 0.0 || time >= needle.inject_until) return;
        emit_accum += needle.flow_rate * dt / pv;
        double count = std::floor(emit_accum);
        size_t n = (size_t)count;
        emit_accum -= count;
        if (n == 0) return;
        V3 axis = normalize_or_zero(needle.axis);
        V3 e1, e2;
        orthonormal_basis(axis, e1, e2);
        double speed = needle.jet_speed();
        V3 v = axis * speed;
        for (size_t q = 0; q < n; ++q) {
            double r = needle.radius * std::sqrt(rng.unit());
            double theta = 2.0 * M_PI * rng.unit();
            double along = (rng.unit() - 0.5) * grid.dx;
            V3 p = needle.tip + e1 * (r * std::cos(theta)) + e2 * (r * std::sin(theta)) + axis * along;
            pos.push_back(p);
            vel.push_back(v);
        }
    }

    void classify() {  // solver.rs:342-371
        size_t nx = grid.nx, ny = grid.ny, nz = grid.nz;
        for (size_t k = 0; k < nz; ++k)
            for (size_t j = 0; j < ny; ++j)
                for (size_t i = 0; i < nx; ++i) {
                    size_t c = (k * ny + j) * nx + i;
                    bool out = has_outlet && outlet.contains(grid.cell_center(i, j, k));
                    cells[c] = out ? AIR : (!cavity_mask[c] ? SOLID : AIR);
                }
        for (V3 p : pos) {
            size_t i, j, k;
            if (cell_of(p, i, j, k)) {
                size_t c = (k * ny + j) * nx + i;
                if (cells[c] == AIR && !in_outlet(p)) cells[c] = FLUID;
            }
        }
    }

    std::vector<double> volume_source(double dt) const {  // solver.rs:392-423
        size_t nx = grid.nx, ny = grid.ny, nz = grid.nz, n = nx * ny * nz;
        double k_vol = fluid.volume_stiffness;
        if (k_vol <= 0.0 || dt <= 0.0) return std::vector<double>(n, 0.0);
        std::vector<uint32_t> count(n, 0);
        for (V3 p : pos) {
            size_t i, j, k;
            if (cell_of(p, i, j, k)) {
                size_t c = (k * ny + j) * nx + i;
                if (cells[c] == FLUID) count[c] += 1;
            }
        }
        double rest = (double)std::max<size_t>(fluid.ppc, 1);
        double unit = grid.dx / dt;
        double cap = VC_MAX_FRACTION * unit;
        std::vector<double> source(n, 0.0);
        for (size_t c = 0; c < n; ++c) {
            if (cells[c] != FLUID) continue;
            double over = (double)count[c] / rest - 1.0;
            if (over > 0.0) source[c] = fmin_(k_vol * over * unit, cap);
        }
        return source;
    }

    V3 project_inside(V3 p) const {  // solver.rs:717-732
        double margin = 0.5 * grid.dx;
        for (int it = 0; it < 3; ++it) {
            double phi = solid.sample(p);
            if (phi <= -margin) break;
            V3 g = normalize_or_zero(solid.gradient(p));
            if (length(g) == 0.0) break;
            p -= g * (phi + margin);
        }
        return p;
    }

    void redistribute() {  // solver.rs:454-557
        size_t nx = grid.nx, ny = grid.ny, nz = grid.nz, ncells = nx * ny * nz;
        size_t target = std::max<size_t>(fluid.ppc, 1);
        uint32_t cap = (uint32_t)std::ceil(fmax_(fluid.redist_cap_factor, 1.0) * (double)target);
        V3 gdir = normalize_or_zero(fluid.gravity);
        std::vector<uint32_t> count(ncells, 0);
        for (size_t sweep = 0; sweep < REDIST_SWEEPS; ++sweep) {
            std::fill(count.begin(), count.end(), 0);
            for (V3 p : pos) {
                size_t i, j, k;
                if (cell_of(p, i, j, k)) count[(k * ny + j) * nx + i] += 1;
            }
            for (size_t idx = 0; idx < pos.size(); ++idx) {
                size_t i, j, k;
                if (!cell_of(pos[idx], i, j, k)) continue;
                size_t c = (k * ny + j) * nx + i;
                if (count[c] <= cap) continue;
                size_t nc_[6];
                double down[6];
                int nn = 0;
                auto add = [&](size_t ncell, V3 dir) {
                    nc_[nn] = ncell;
                    down[nn] = dot(dir, gdir);
                    ++nn;
                };
                if (i > 0) add(c - 1, v3(-1, 0, 0));
                if (i + 1 < nx) add(c + 1, v3(1, 0, 0));
                if (j > 0) add(c - nx, v3(0, -1, 0));
                if (j + 1 < ny) add(c + nx, v3(0, 1, 0));
                if (k > 0) add(c - nx * ny, v3(0, 0, -1));
                if (k + 1 < nz) add(c + nx * ny, v3(0, 0, 1));
                bool have = false;
                size_t best = 0;
                double best_down = -std::numeric_limits<double>::infinity();
                uint32_t best_room = 0;
                for (int q = 0; q < nn; ++q) {
                    size_t ncell = nc_[q];
                    if (!cavity_mask[ncell] || count[ncell] >= cap) continue;
                    uint32_t room = cap - count[ncell];
                    bool better = !have || down[q] > best_down ||
                                  (down[q] == best_down && room > best_room);
                    if (better) {
                        have = true;
                        best = ncell;
                        best_down = down[q];
                        best_room = room;
                    }
                }
                if (have) {
                    count[c] -= 1;
                    count[best] += 1;
                    size_t ci = best % nx, cj = (best / nx) % ny, ck = best / (nx * ny);
                    V3 jit = hash_jitter((uint64_t)idx);
                    V3 p = grid.cell_center(ci, cj, ck) + jit * grid.dx;
                    p = project_inside(p);
                    pos[idx] = p;
                    vel[idx] = grid.velocity_at(p);
                }
            }
        }
    }

    void p2g() {  // solver.rs:560-585
        std::fill(grid.u.begin(), grid.u.end(), 0.0);
        std::fill(grid.v.begin(), grid.v.end(), 0.0);
        std::fill(grid.w.begin(), grid.w.end(), 0.0);
        std::vector<double> wu(grid.u.size(), 0.0), wv(grid.v.size(), 0.0), ww(grid.w.size(), 0.0);
        for (size_t q = 0; q < pos.size(); ++q) {
            double gx, gy, gz;
            grid.u_coords(pos[q], gx, gy, gz);
            trilinear_scatter(grid.u.data(), wu.data(), grid.ud(), gx, gy, gz, vel[q].x);
            grid.v_coords(pos[q], gx, gy, gz);
            trilinear_scatter(grid.v.data(), wv.data(), grid.vd(), gx, gy, gz, vel[q].y);
            grid.w_coords(pos[q], gx, gy, gz);
            trilinear_scatter(grid.w.data(), ww.data(), grid.wd(), gx, gy, gz, vel[q].z);
        }
        auto normalize = [](std::vector<double>& f, const std::vector<double>& w) {  // solver.rs:944-952
            for (size_t i = 0; i < f.size(); ++i) f[i] = w[i] > 1e-12 ? f[i] / w[i] : 0.0;
        };
        normalize(grid.u, wu);
        normalize(grid.v, wv);
        normalize(grid.w, ww);
    }

    void add_forces(double dt) {  // solver.rs:593-604
        V3 g = fluid.gravity;
        if (g.x != 0.0) for (double& x : grid.u) x += g.x * dt;
        if (g.y != 0.0) for (double& x : grid.v) x += g.y * dt;
        if (g.z != 0.0) for (double& x : grid.w) x += g.z * dt;
    }

    static void extrapolate(std::vector<double>& field, const std::vector<uint8_t>& valid, Dims d,
                            int iters) {  // solver.rs:960-1009
        size_t nx = d.nx, ny = d.ny, nz = d.nz;
        auto idx = [&](size_t i, size_t j, size_t k) { return (k * ny + j) * nx + i; };
        std::vector<uint8_t> known = valid;
        for (int it = 0; it < iters; ++it) {
            std::vector<double> snap = field;
            std::vector<uint8_t> ks = known;
            for (size_t k = 0; k < nz; ++k)
                for (size_t j = 0; j < ny; ++j)
                    for (size_t i = 0; i < nx; ++i) {
                        size_t c = idx(i, j, k);
                        if (ks[c]) continue;
                        double sum = 0.0;
                        int cnt = 0;
                        auto acc = [&](size_t ci, size_t cj, size_t ck) {
                            size_t n = idx(ci, cj, ck);
                            if (ks[n]) { sum += snap[n]; ++cnt; }
                        };
                        if (i > 0) acc(i - 1, j, k);
                        if (i + 1 < nx) acc(i + 1, j, k);
                        if (j > 0) acc(i, j - 1, k);
                        if (j + 1 < ny) acc(i, j + 1, k);
                        if (k > 0) acc(i, j, k - 1);
                        if (k + 1 < nz) acc(i, j, k + 1);
                        if (cnt > 0) {
                            field[c] = sum / (double)cnt;
                            known[c] = 1;
                        }
                    }
        }
    }

    void extrapolate_velocities() {  // solver.rs:608-647
        size_t nx = grid.nx, ny = grid.ny, nz = grid.nz;
        auto fl = [&](size_t i, size_t j, size_t k) { return cells[(k * ny + j) * nx + i] == FLUID; };
        std::vector<uint8_t> vu(grid.u.size(), 0), vv(grid.v.size(), 0), vw(grid.w.size(), 0);
        for (size_t k = 0; k < nz; ++k)
            for (size_t j = 0; j < ny; ++j)
                for (size_t i = 0; i <= nx; ++i)
                    vu[grid.u_idx(i, j, k)] = (i > 0 && fl(i - 1, j, k)) || (i < nx && fl(i, j, k));
        for (size_t k = 0; k < nz; ++k)
            for (size_t j = 0; j <= ny; ++j)
                for (size_t i = 0; i < nx; ++i)
                    vv[grid.v_idx(i, j, k)] = (j > 0 && fl(i, j - 1, k)) || (j < ny && fl(i, j, k));
        for (size_t k = 0; k <= nz; ++k)
            for (size_t j = 0; j < ny; ++j)
                for (size_t i = 0; i < nx; ++i)
                    vw[grid.w_idx(i, j, k)] = (k > 0 && fl(i, j, k - 1)) || (k < nz && fl(i, j, k));
        extrapolate(grid.u, vu, grid.ud(), 4);
        extrapolate(grid.v, vv, grid.vd(), 4);
        extrapolate(grid.w, vw, grid.wd(), 4);
    }

    void g2p() {  // solver.rs:650-677
        double flip = clampd(fluid.flip_ratio, 0.0, 1.0);
        std::vector<double> du(grid.u.size()), dv(grid.v.size()), dw(grid.w.size());
        for (size_t i = 0; i < du.size(); ++i) du[i] = grid.u[i] - saved_u[i];
        for (size_t i = 0; i < dv.size(); ++i) dv[i] = grid.v[i] - saved_v[i];
        for (size_t i = 0; i < dw.size(); ++i) dw[i] = grid.w[i] - saved_w[i];
        for (size_t q = 0; q < pos.size(); ++q) {
            V3 p = pos[q];
            V3 pic = grid.velocity_at(p);
            double gx, gy, gz;
            grid.u_coords(p, gx, gy, gz);
            double dvx = trilinear_sample(du.data(), grid.ud(), gx, gy, gz);
            grid.v_coords(p, gx, gy, gz);
            double dvy = trilinear_sample(dv.data(), grid.vd(), gx, gy, gz);
            grid.w_coords(p, gx, gy, gz);
            double dvz = trilinear_sample(dw.data(), grid.wd(), gx, gy, gz);
            V3 flip_v = vel[q] + v3(dvx, dvy, dvz);
            vel[q] = flip_v * flip + pic * (1.0 - flip);
        }
    }

    void advect(double dt) {  // solver.rs:693-711
        double max_step = grid.dx;
        for (size_t q = 0; q < pos.size(); ++q) {
            V3 p0 = pos[q];
            V3 v0 = grid.velocity_at(p0);
            V3 mid = p0 + v0 * (0.5 * dt);
            V3 vmid = grid.velocity_at(mid);
            V3 st = vmid * dt;
            double len = length(st);
            if (len > max_step) st = st * (max_step / len);
            V3 p = project_inside(p0 + st);
            pos[q] = solid.sample(p) <= 0.0 ? p : p0;
        }
    }

    void enforce_particle_bounds() {  // solver.rs:736-755, particles.rs:38-49
        Aabb bb = solid.bounds();
        uint64_t dr = 0;
        size_t w = 0;
        for (size_t r = 0; r < pos.size(); ++r) {
            V3 p = pos[r];
            bool keep;
            if (!bb.contains(p)) keep = false;
            else if (has_outlet && outlet.contains(p)) { ++dr; keep = false; }
            else keep = solid.sample(p) < 0.5 * solid.dx;
            if (keep) {
                pos[w] = pos[r];
                vel[w] = vel[r];
                ++w;
            }
        }
        pos.resize(w);
        vel.resize(w);
        drained += dr;
    }

    double max_pressure() const {  // solver.rs:859-866
        double m = 0.0;
        for (size_t c = 0; c < cells.size(); ++c)
            if (cells[c] == FLUID) m = fmax_(m, pressure[c]);
        return m;
    }
    double mean_pressure() const {  // solver.rs:869-881
        double s = 0.0;
        uint64_t n = 0;
        for (size_t c = 0; c < cells.size(); ++c)
            if (cells[c] == FLUID) { s = s + pressure[c]; n += 1; }
        return n > 0 ? s / (double)n : 0.0;
    }
    double max_speed() const {  // solver.rs:884-890
        double m = 0.0;
        for (V3 v : vel) m = fmax_(m, length(v));
        return m;
    }
    double kinetic_energy() const {  // particles.rs:52-56
        double s = -0.0;
        for (V3 v : vel) s += length_sq(v);
        return 0.5 * s;
    }
};

struct orc_metrics {  // metrics.rs:102-114
    double cavity_volume;
    size_t nx, ny, nz;
    V3 origin;
    double dx;
    std::vector<uint8_t> is_wall, washed;
    size_t wall_count;
    std::vector<orc_frame_metrics> history;
    double injected_ml;

    bool cell_index(V3 p, size_t& c) const {  // metrics.rs:434-445
        V3 l = (p - origin) / dx;
        if (l.x < 0.0 || l.y < 0.0 || l.z < 0.0) return false;
        double mx = 1.8e19;
        size_t i = l.x >= mx ? SIZE_MAX : (size_t)l.x;
        size_t j = l.y >= mx ? SIZE_MAX : (size_t)l.y;
        size_t k = l.z >= mx ? SIZE_MAX : (size_t)l.z;
        if (i < nx && j < ny && k < nz) {
            c = (k * ny + j) * nx + i;
            return true;
        }
        return false;
    }
};

namespace {
const double M3_TO_ML = 1.0e6;               // metrics.rs:23
const double PA_TO_MMHG = 1.0 / 133.322;     // metrics.rs:24
const double MEMBRANE_PRESSURE_CAP_FACTOR = 3.0;  // metrics.rs:454

void membrane_stats(const std::vector<double>& values, double cap, double& mean, double& peak,
                    uint64_t& artifacts) {  // metrics.rs:460-478
    double sum = 0.0;
    peak = 0.0;
    uint64_t n = 0;
    artifacts = 0;
    for (double p : values) {
        if (p > cap) { ++artifacts; continue; }
        sum += p;
        peak = fmax_(peak, p);
        ++n;
    }
    if (n == 0) { mean = 0.0; peak = 0.0; }
    else mean = sum / (double)n;
}
}  // namespace

// ================================================================= C ABI
// ---------------------------------------------------------------- render.rs
// render_slice / render_timeseries (render.rs:139-415) into an RGB8 buffer.
namespace {

const uint8_t RC_BG[3] = {18, 18, 22};        // render.rs:22-25
const uint8_t RC_INTERIOR[3] = {232, 236, 244};
const uint8_t RC_WALL[3] = {44, 44, 54};
const uint8_t RC_NEEDLE[3] = {255, 80, 80};
const uint8_t RC_FILM[3] = {242, 178, 92};     // render.rs:31-32
const uint8_t RC_DEEP[3] = {150, 78, 18};

struct Rgb8 {
    uint32_t w, h;
    uint8_t* px;
    void set(uint32_t x, uint32_t y, const uint8_t c[3]) { std::memcpy(px + 3 * ((size_t)y * w + x), c, 3); }
    void put(int64_t x, int64_t y, const uint8_t c[3]) {  // render.rs:430-434
        if (x >= 0 && y >= 0 && (uint64_t)x < w && (uint64_t)y < h) set((uint32_t)x, (uint32_t)y, c);
    }
};

int64_t as_i64(double f) {  // Rust `as i64`: truncation, saturating, NaN -> 0
    if (std::isnan(f)) return 0;
    if (f >= 9223372036854775807.0) return INT64_MAX;
    if (f <= -9223372036854775808.0) return INT64_MIN;
    return (int64_t)f;
}
uint8_t as_u8(double f) {  // Rust `as u8`
    if (std::isnan(f) || f <= 0.0) return 0;
    if (f >= 255.0) return 255;
    return (uint8_t)f;
}
double clamp01(double t) { return t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t); }

void r_disk(Rgb8& im, int64_t cx, int64_t cy, int64_t r, const uint8_t c[3]) {  // render.rs:436-444
    for (int64_t dy = -r; dy <= r; ++dy)
        for (int64_t dx = -r; dx <= r; ++dx)
            if (dx * dx + dy * dy <= r * r) im.put(cx + dx, cy + dy, c);
}

void r_line(Rgb8& im, int64_t x0, int64_t y0, int64_t x1, int64_t y1, const uint8_t c[3]) {  // render.rs:447-468
    int64_t dx = x1 - x0 < 0 ? x0 - x1 : x1 - x0;
    int64_t dy = -(y1 - y0 < 0 ? y0 - y1 : y1 - y0);
    int64_t sx = x0 < x1 ? 1 : -1, sy = y0 < y1 ? 1 : -1;
    int64_t err = dx + dy;
    for (;;) {
        im.put(x0, y0, c);
        if (x0 == x1 && y0 == y1) break;
        int64_t e2 = 2 * err;
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

uint8_t r_lerp(uint8_t a, uint8_t b, double t) {  // render.rs:311-316
    t = clamp01(t);
    double v = std::round((double)a * (1.0 - t) + (double)b * t);
    v = v < 0.0 ? 0.0 : (v > 255.0 ? 255.0 : v);
    return (uint8_t)v;
}

void r_speed(double t, uint8_t c[3]) {  // render.rs:417-428
    t = clamp01(t);
    double r, g, b;
    if (t < 0.5) {
        double u = t / 0.5;
        r = 0.0; g = u; b = 1.0 - u;
    } else {
        double u = (t - 0.5) / 0.5;
        r = u; g = 1.0 - u; b = 0.0;
    }
    c[0] = as_u8(r * 255.0);
    c[1] = as_u8(g * 255.0);
    c[2] = as_u8(b * 255.0);
}

double comp(V3 a, int axis) { return axis == 0 ? a.x : (axis == 1 ? a.y : a.z); }

}  // namespace

static void slice_dims(const orc_solver& s, const orc_slice_plane& p, uint32_t target, uint32_t& w, uint32_t& h,
                       double mn[3], double mx[3], double& wm, double& hm) {  // render.rs:139-156
    Aabb bb = s.solid.bounds();
    mn[0] = bb.min.x; mn[1] = bb.min.y; mn[2] = bb.min.z;
    mx[0] = bb.max.x; mx[1] = bb.max.y; mx[2] = bb.max.z;
    wm = fmax_(mx[p.hax] - mn[p.hax], 1e-9);
    hm = fmax_(mx[p.vax] - mn[p.vax], 1e-9);
    uint32_t t = target > 1 ? target : 1;
    if (wm >= hm) {
        w = t;
        h = (uint32_t)fmax_(std::round((double)target * hm / wm), 1.0);
    } else {
        w = (uint32_t)fmax_(std::round((double)target * wm / hm), 1.0);
        h = t;
    }
}

extern "C" {

void orc_set_threads(int n) { g_threads = n; }
int orc_get_threads(void) { return nthreads(); }

double orc_point_triangle_distance_sq(const double p[3], const double a[3], const double b[3],
                                      const double c[3]) {
    return point_triangle_distance_sq(from(p), from(a), from(b), from(c));
}

double orc_signed_distance_to_mesh(const double p[3], const double* tris, size_t ntri) {
    return signed_distance_to_mesh(from(p), tris, ntri);
}

void orc_sdf_mesh_grid(const double* tris, size_t ntri, double dx, double padding,
                       double origin[3], uint64_t dims[3]) {  // sdf.rs:47-58
    Aabb bb = Aabb::empty();
    for (size_t q = 0; q < 3 * ntri; ++q) bb.expand(from(tris + 3 * q));
    bb = bb.padded(padding);
    V3 size = bb.size();
    dims[0] = (uint64_t)std::ceil(size.x / dx) + 1;
    dims[1] = (uint64_t)std::ceil(size.y / dx) + 1;
    dims[2] = (uint64_t)std::ceil(size.z / dx) + 1;
    to(bb.min, origin);
}

void orc_sdf_from_mesh(const double* tris, size_t ntri, const double origin[3], double dx,
                       const uint64_t dims[3], double* out) {  // sdf.rs:53-86
    size_t nx = dims[0], ny = dims[1], nz = dims[2];
    V3 o = from(origin);
    parallel_for(nz, [&](size_t k0, size_t k1) {
        for (size_t k = k0; k < k1; ++k)
            for (size_t j = 0; j < ny; ++j)
                for (size_t i = 0; i < nx; ++i) {
                    V3 p = o + v3((double)i * dx, (double)j * dx, (double)k * dx);
                    out[(k * ny + j) * nx + i] = signed_distance_to_mesh(p, tris, ntri);
                }
    }, nx * ny * nz * 64);
}

double orc_sinus_implicit(const orc_sinus* s, const double p[3]) {
    return to_sinus(s).implicit(from(p));
}

void orc_sinus_bounds(const orc_sinus* s, double mn[3], double mx[3]) {
    Aabb bb = to_sinus(s).bounds();
    to(bb.min, mn);
    to(bb.max, mx);
}

double orc_sinus_socket_bottom_y(const orc_sinus* s) { return to_sinus(s).socket_bottom_y(); }

void orc_sinus_suggested_needle(const orc_sinus* s, double tip[3], double axis[3]) {  // sinus.rs:154-160
    Sinus q = to_sinus(s);
    to(v3(q.sx, q.socket_top_y() + q.semi_axes.y * 0.15, q.sz), tip);
    to(v3(0, 1, 0), axis);
}

void orc_sdf_from_sinus(const orc_sinus* s, const double origin[3], double dx,
                        const uint64_t dims[3], double* out) {  // sdf.rs:90-116
    Sinus q = to_sinus(s);
    size_t nx = dims[0], ny = dims[1], nz = dims[2];
    V3 o = from(origin);
    parallel_for(nz, [&](size_t k0, size_t k1) {
        for (size_t k = k0; k < k1; ++k)
            for (size_t j = 0; j < ny; ++j)
                for (size_t i = 0; i < nx; ++i)
                    out[(k * ny + j) * nx + i] =
                        q.implicit(o + v3((double)i * dx, (double)j * dx, (double)k * dx));
    }, nx * ny * nz * 64);
}

double orc_sinus_mesh_volume(const orc_sinus* s, uint64_t* ntri_out) {
    std::vector<V3> verts;
    std::vector<uint32_t> idx;
    sinus_mesh(to_sinus(s), verts, idx);
    if (ntri_out) *ntri_out = idx.size() / 3;
    return std::fabs(signed_volume(verts, idx));
}

size_t orc_sinus_mesh(const orc_sinus* s, double* tris_out, size_t cap_tris) {
    std::vector<V3> verts;
    std::vector<uint32_t> idx;
    sinus_mesh(to_sinus(s), verts, idx);
    size_t nt = idx.size() / 3;
    if (tris_out && cap_tris >= nt)
        for (size_t t = 0; t < nt; ++t)
            for (int c = 0; c < 3; ++c) to(verts[idx[3 * t + c]], tris_out + 9 * t + 3 * c);
    return nt;
}

double orc_mesh_signed_volume(const double* tris, size_t ntri) {
    double v = 0.0;
    for (size_t t = 0; t < ntri; ++t) {
        V3 a = from(tris + 9 * t), b = from(tris + 9 * t + 3), c = from(tris + 9 * t + 6);
        v += dot(a, cross(b, c)) / 6.0;
    }
    return v;
}

static Sdf make_sdf(const double* data, const uint64_t dims[3], const double origin[3], double dx) {
    Sdf s;
    s.origin = from(origin);
    s.dx = dx;
    s.nx = dims[0]; s.ny = dims[1]; s.nz = dims[2];
    s.data.assign(data, data + s.nx * s.ny * s.nz);
    return s;
}

double orc_sdf_sample(const double* data, const uint64_t dims[3], const double origin[3],
                      double dx, const double p[3]) {
    return make_sdf(data, dims, origin, dx).sample(from(p));
}

void orc_sdf_gradient(const double* data, const uint64_t dims[3], const double origin[3],
                      double dx, const double p[3], double g[3]) {
    to(make_sdf(data, dims, origin, dx).gradient(from(p)), g);
}

orc_solver* orc_solver_new(const double* sdf_data, const uint64_t sdf_dims[3],
                           const double sdf_origin[3], double sdf_dx, double sim_dx,
                           const orc_fluid* fl, const orc_needle* nd) {  // solver.rs:184-222
    orc_solver* s = new orc_solver();
    s->solid = make_sdf(sdf_data, sdf_dims, sdf_origin, sdf_dx);
    Aabb bb = s->solid.bounds();
    V3 size = bb.size();
    size_t nx = (size_t)fmax_(std::ceil(size.x / sim_dx), 1.0);
    size_t ny = (size_t)fmax_(std::ceil(size.y / sim_dx), 1.0);
    size_t nz = (size_t)fmax_(std::ceil(size.z / sim_dx), 1.0);
    MacGrid& g = s->grid;
    g.nx = nx; g.ny = ny; g.nz = nz; g.dx = sim_dx; g.origin = bb.min;
    g.u.assign((nx + 1) * ny * nz, 0.0);
    g.v.assign(nx * (ny + 1) * nz, 0.0);
    g.w.assign(nx * ny * (nz + 1), 0.0);
    size_t n = nx * ny * nz;
    s->cavity_mask.resize(n);
    for (size_t c = 0; c < n; ++c) {
        size_t i = c % nx, j = (c / nx) % ny, k = c / (nx * ny);
        s->cavity_mask[c] = s->solid.sample(g.cell_center(i, j, k)) < 0.0;
    }
    s->fluid.density = fl->density;
    s->fluid.gravity = from(fl->gravity);
    s->fluid.flip_ratio = fl->flip_ratio;
    s->fluid.ppc = fl->particles_per_cell;
    s->fluid.volume_stiffness = fl->volume_stiffness;
    s->fluid.redistribute = fl->redistribute != 0;
    s->fluid.redist_cap_factor = fl->redist_cap_factor;
    orc_solver_set_needle(s, nd);
    s->pressure.assign(n, 0.0);
    s->cells.assign(n, AIR);
    return s;
}

void orc_solver_free(orc_solver* s) { delete s; }

void orc_solver_set_needle(orc_solver* s, const orc_needle* nd) {
    s->needle.tip = from(nd->tip);
    s->needle.axis = from(nd->axis);
    s->needle.radius = nd->radius;
    s->needle.flow_rate = nd->flow_rate;
    s->needle.inject_until = nd->inject_until;
}

void orc_solver_set_outlet(orc_solver* s, int has, const double mn[3], const double mx[3]) {
    s->has_outlet = has != 0;
    if (has) s->outlet = Aabb{from(mn), from(mx)};
}

void orc_solver_set_solve(orc_solver* s, uint64_t max_iters, double tol) {
    s->max_iters = max_iters;
    s->tol = tol;
}

void orc_solver_step(orc_solver* s, double dt) { s->step(dt); }
void orc_solver_substep(orc_solver* s, double dt) { s->substep(dt); }
void orc_solver_phase(orc_solver* s, int phase, double dt) { s->phase(phase, dt); }
double orc_solver_cfl_dt(const orc_solver* s) { return s->cfl_dt(); }

void orc_solver_grid(const orc_solver* s, uint64_t dims[3], double origin[3], double* dx) {
    dims[0] = s->grid.nx; dims[1] = s->grid.ny; dims[2] = s->grid.nz;
    to(s->grid.origin, origin);
    *dx = s->grid.dx;
}

size_t orc_solver_num_particles(const orc_solver* s) { return s->pos.size(); }

void orc_solver_get_particles(const orc_solver* s, double* pos, double* vel) {
    for (size_t q = 0; q < s->pos.size(); ++q) {
        if (pos) to(s->pos[q], pos + 3 * q);
        if (vel) to(s->vel[q], vel + 3 * q);
    }
}

void orc_solver_set_particles(orc_solver* s, size_t n, const double* pos, const double* vel) {
    s->pos.resize(n);
    s->vel.resize(n);
    for (size_t q = 0; q < n; ++q) {
        s->pos[q] = from(pos + 3 * q);
        s->vel[q] = from(vel + 3 * q);
    }
}

void orc_solver_get_scalars(const orc_solver* s, double* time, double* emit_accum,
                            uint64_t* steps, uint64_t* last_pcg_iters, uint64_t* last_substeps,
                            uint64_t* drained, uint64_t* rng) {
    if (time) *time = s->time;
    if (emit_accum) *emit_accum = s->emit_accum;
    if (steps) *steps = s->steps;
    if (last_pcg_iters) *last_pcg_iters = s->last_pcg_iters;
    if (last_substeps) *last_substeps = s->last_substeps;
    if (drained) *drained = s->drained;
    if (rng) *rng = s->rng.s;
}

void orc_solver_set_scalars(orc_solver* s, double time, double emit_accum, uint64_t steps,
                            uint64_t drained, uint64_t rng) {
    s->time = time;
    s->emit_accum = emit_accum;
    s->steps = steps;
    s->drained = drained;
    s->rng.s = rng;
}

static std::vector<double>* face_ptr(orc_solver* s, int which) {
    switch (which) {
        case 0: return &s->grid.u;
        case 1: return &s->grid.v;
        case 2: return &s->grid.w;
        case 3: return &s->saved_u;
        case 4: return &s->saved_v;
        case 5: return &s->saved_w;
    }
    return nullptr;
}

void orc_solver_get_face(const orc_solver* s, int which, double* out) {
    const std::vector<double>* f = face_ptr(const_cast<orc_solver*>(s), which);
    if (f) std::memcpy(out, f->data(), f->size() * sizeof(double));
}

void orc_solver_set_face(orc_solver* s, int which, const double* in) {
    std::vector<double>* f = face_ptr(s, which);
    if (!f) return;
    size_t n = (which % 3 == 0) ? s->grid.u.size() : (which % 3 == 1) ? s->grid.v.size() : s->grid.w.size();
    f->assign(in, in + n);
}

void orc_solver_get_cells(const orc_solver* s, uint8_t* out) {
    std::memcpy(out, s->cells.data(), s->cells.size());
}
void orc_solver_set_cells(orc_solver* s, const uint8_t* in) {
    std::memcpy(s->cells.data(), in, s->cells.size());
}
void orc_solver_get_cavity_mask(const orc_solver* s, uint8_t* out) {
    std::memcpy(out, s->cavity_mask.data(), s->cavity_mask.size());
}
void orc_solver_get_pressure(const orc_solver* s, double* out) {
    std::memcpy(out, s->pressure.data(), s->pressure.size() * sizeof(double));
}
void orc_solver_get_source(const orc_solver* s, double dt, double* out) {
    std::vector<double> src = s->volume_source(dt);
    std::memcpy(out, src.data(), src.size() * sizeof(double));
}
double orc_solver_max_pressure(const orc_solver* s) { return s->max_pressure(); }
double orc_solver_mean_pressure(const orc_solver* s) { return s->mean_pressure(); }
double orc_solver_max_speed(const orc_solver* s) { return s->max_speed(); }
double orc_solver_kinetic_energy(const orc_solver* s) { return s->kinetic_energy(); }
double orc_solver_grid_max_speed(const orc_solver* s) { return s->grid.max_speed(); }

uint64_t orc_solver_max_particles_per_cell(const orc_solver* s) {  // solver.rs:770-782
    std::vector<uint32_t> count(s->grid.nx * s->grid.ny * s->grid.nz, 0);
    uint32_t mx = 0;
    for (V3 p : s->pos) {
        size_t i, j, k;
        if (s->cell_of(p, i, j, k)) {
            size_t c = (k * s->grid.ny + j) * s->grid.nx + i;
            count[c] += 1;
            mx = std::max(mx, count[c]);
        }
    }
    return mx;
}

uint64_t orc_solver_cells_fluid_count(const orc_solver* s) {
    uint64_t n = 0;
    for (uint8_t c : s->cells) n += (c == FLUID);
    return n;
}

void orc_solver_phase_times(const orc_solver* s, double out[12]) {
    for (int q = 0; q < 12; ++q) out[q] = s->phase_t[q];
}

uint64_t orc_project(uint64_t nx, uint64_t ny, uint64_t nz, double dx, double* u, double* v,
                     double* w, const uint8_t* cells, double rho, double dt, uint64_t max_iters,
                     double tol, const double* source, double* pressure_out,
                     double* residual_out) {
    MacGrid g;
    g.nx = nx; g.ny = ny; g.nz = nz; g.dx = dx; g.origin = v3(0, 0, 0);
    g.u.assign(u, u + (nx + 1) * ny * nz);
    g.v.assign(v, v + nx * (ny + 1) * nz);
    g.w.assign(w, w + nx * ny * (nz + 1));
    PcgResult rep = project_with_source(g, cells, rho, dt, max_iters, tol, source);
    std::memcpy(u, g.u.data(), g.u.size() * sizeof(double));
    std::memcpy(v, g.v.data(), g.v.size() * sizeof(double));
    std::memcpy(w, g.w.data(), g.w.size() * sizeof(double));
    if (pressure_out) std::memcpy(pressure_out, rep.pressure.data(), rep.pressure.size() * sizeof(double));
    if (residual_out) *residual_out = rep.residual;
    return rep.iters;
}

static Laplacian assemble(uint64_t nx, uint64_t ny, uint64_t nz, const uint8_t* cells) {
    Laplacian a;
    a.nx = nx; a.ny = ny; a.nz = nz;
    size_t n = nx * ny * nz;
    a.diag.assign(n, 0.0); a.plus_x.assign(n, 0.0); a.plus_y.assign(n, 0.0); a.plus_z.assign(n, 0.0);
    auto cell = [&](size_t i, size_t j, size_t k) { return cells[(k * ny + j) * nx + i]; };
    for (size_t k = 0; k < nz; ++k)
        for (size_t j = 0; j < ny; ++j)
            for (size_t i = 0; i < nx; ++i) {
                size_t c = (k * ny + j) * nx + i;
                if (cells[c] != FLUID) continue;
                double diag = 0.0;
                auto consider = [&](int64_t ni, int64_t nj, int64_t nk, double* plus) {
                    bool inside = ni >= 0 && nj >= 0 && nk >= 0 && (size_t)ni < nx &&
                                  (size_t)nj < ny && (size_t)nk < nz;
                    uint8_t kind = inside ? cell(ni, nj, nk) : SOLID;
                    if (kind == AIR) diag += 1.0;
                    else if (kind == FLUID) { diag += 1.0; if (plus) *plus = -1.0; }
                };
                int64_t ii = i, jj = j, kk = k;
                consider(ii - 1, jj, kk, nullptr);
                consider(ii + 1, jj, kk, &a.plus_x[c]);
                consider(ii, jj - 1, kk, nullptr);
                consider(ii, jj + 1, kk, &a.plus_y[c]);
                consider(ii, jj, kk - 1, nullptr);
                consider(ii, jj, kk + 1, &a.plus_z[c]);
                a.diag[c] = diag;
            }
    return a;
}

void orc_build_mic0(uint64_t nx, uint64_t ny, uint64_t nz, const uint8_t* cells, double* precon) {
    Laplacian a = assemble(nx, ny, nz, cells);
    std::vector<double> p = build_mic0(a, cells);
    std::memcpy(precon, p.data(), p.size() * sizeof(double));
}

void orc_apply_mic0(uint64_t nx, uint64_t ny, uint64_t nz, const uint8_t* cells,
                    const double* precon, const double* r, double* z) {
    Laplacian a = assemble(nx, ny, nz, cells);
    std::vector<double> pc(precon, precon + nx * ny * nz), q(nx * ny * nz, 0.0);
    apply_mic0(a, pc, cells, r, z, q);
}

double orc_dot(const double* a, const double* b, size_t n) { return dot_det(a, b, n); }

orc_metrics* orc_metrics_new(const orc_solver* s, double cavity_volume) {  // metrics.rs:119-185
    orc_metrics* m = new orc_metrics();
    const MacGrid& g = s->grid;
    size_t nx = g.nx, ny = g.ny, nz = g.nz, n = nx * ny * nz;
    m->cavity_volume = cavity_volume;
    m->nx = nx; m->ny = ny; m->nz = nz; m->origin = g.origin; m->dx = g.dx;
    std::vector<uint8_t> inside(n, 0);
    for (size_t k = 0; k < nz; ++k)
        for (size_t j = 0; j < ny; ++j)
            for (size_t i = 0; i < nx; ++i)
                inside[(k * ny + j) * nx + i] = s->solid.sample(g.cell_center(i, j, k)) < 0.0;
    m->is_wall.assign(n, 0);
    m->wall_count = 0;
    for (size_t k = 0; k < nz; ++k)
        for (size_t j = 0; j < ny; ++j)
            for (size_t i = 0; i < nx; ++i) {
                size_t c = (k * ny + j) * nx + i;
                if (!inside[c]) continue;
                auto nb_solid = [&](int64_t ci, int64_t cj, int64_t ck) {
                    if (ci < 0 || cj < 0 || ck < 0 || (size_t)ci >= nx || (size_t)cj >= ny ||
                        (size_t)ck >= nz)
                        return true;
                    return !inside[((size_t)ck * ny + (size_t)cj) * nx + (size_t)ci];
                };
                int64_t ii = i, jj = j, kk = k;
                bool touches = nb_solid(ii - 1, jj, kk) || nb_solid(ii + 1, jj, kk) ||
                               nb_solid(ii, jj - 1, kk) || nb_solid(ii, jj + 1, kk) ||
                               nb_solid(ii, jj, kk - 1) || nb_solid(ii, jj, kk + 1);
                if (touches) {
                    m->is_wall[c] = 1;
                    m->wall_count += 1;
                }
            }
    m->washed.assign(n, 0);
    m->injected_ml = 0.0;
    return m;
}

void orc_metrics_free(orc_metrics* m) { delete m; }

void orc_metrics_record(orc_metrics* m, const orc_solver* s, uint64_t frame,
                        orc_frame_metrics* out) {  // metrics.rs:188-316
    std::set<size_t> wet_wall;
    for (V3 p : s->pos) {
        size_t c;
        if (m->cell_index(p, c) && m->is_wall[c]) {
            m->washed[c] = 1;
            wet_wall.insert(c);
        }
    }
    size_t washed_count = 0;
    for (uint8_t b : m->washed) washed_count += b;
    double wall_coverage = m->wall_count > 0 ? (double)washed_count / (double)m->wall_count : 0.0;
    double fluid_volume = s->fluid_volume();
    double drained_volume = s->drained_volume();
    double fill_fraction = m->cavity_volume > 0.0 ? fluid_volume / m->cavity_volume : 0.0;
    double max_p = s->max_pressure();
    m->injected_ml = (fluid_volume + drained_volume) * M3_TO_ML;
    double v_jet = s->needle.jet_speed();
    double stagnation = 0.5 * s->fluid.density * v_jet * v_jet;
    double hydrostatic = s->fluid.density * length(s->fluid.gravity) * ((double)m->ny * m->dx);
    double p_cap = MEMBRANE_PRESSURE_CAP_FACTOR * stagnation + hydrostatic + 500.0;
    std::vector<double> wall_p;
    wall_p.reserve(wet_wall.size());
    for (size_t c : wet_wall) wall_p.push_back(s->pressure[c]);
    double wall_mean, wall_peak;
    uint64_t artifacts;
    membrane_stats(wall_p, p_cap, wall_mean, wall_peak, artifacts);
    orc_frame_metrics f;
    f.frame = frame;
    f.time_s = s->time;
    f.particles = s->pos.size();
    f.fluid_volume_ml = fluid_volume * M3_TO_ML;
    f.drained_volume_ml = drained_volume * M3_TO_ML;
    f.fill_fraction = fill_fraction;
    f.wall_coverage = wall_coverage;
    f.mean_pressure_pa = s->mean_pressure();
    f.max_pressure_pa = max_p;
    f.max_pressure_mmhg = max_p * PA_TO_MMHG;
    f.wall_pressure_pa = wall_mean;
    f.peak_wall_pressure_pa = wall_peak;
    f.peak_wall_pressure_mmhg = wall_peak * PA_TO_MMHG;
    f.membrane_artifacts = artifacts;
    f.max_speed_m_s = s->max_speed();
    f.kinetic_energy = s->kinetic_energy();
    f.pcg_iters = s->last_pcg_iters;
    m->history.push_back(f);
    if (out) *out = f;
}

void orc_metrics_summary(const orc_metrics* m, orc_summary* out) {  // metrics.rs:324-382
    double peak_fill = 0.0, peak_cov = 0.0, peak_p = 0.0, peak_membrane = 0.0;
    for (const auto& f : m->history) {
        peak_fill = fmax_(peak_fill, f.fill_fraction);
        peak_cov = fmax_(peak_cov, f.wall_coverage);
        peak_p = fmax_(peak_p, f.max_pressure_pa);
        peak_membrane = fmax_(peak_membrane, f.peak_wall_pressure_pa);
    }
    double mean_membrane = 0.0;
    if (!m->history.empty()) {
        double s = -0.0;
        for (const auto& f : m->history) s += f.wall_pressure_pa;
        mean_membrane = s / (double)m->history.size();
    }
    uint64_t artifacts_total = 0;
    for (const auto& f : m->history) artifacts_total += f.membrane_artifacts;
    const orc_frame_metrics* last = m->history.empty() ? nullptr : &m->history.back();
    double final_fill = last ? last->fill_fraction : 0.0;
    double final_cov = last ? last->wall_coverage : 0.0;
    double final_time = last ? last->time_s : 0.0;
    double resident_ml = last ? last->fluid_volume_ml : 0.0;
    double drained_ml = last ? last->drained_volume_ml : 0.0;
    double injected = resident_ml + drained_ml;
    double mass_balance = m->injected_ml > 0.0 ? injected / m->injected_ml : 1.0;
    orc_summary s;
    s.frames = m->history.size();
    s.final_time_s = final_time;
    s.peak_fill_fraction = peak_fill;
    s.final_fill_fraction = final_fill;
    s.peak_wall_coverage = peak_cov;
    s.final_wall_coverage = final_cov;
    s.peak_membrane_pressure_pa = peak_membrane;
    s.peak_membrane_pressure_mmhg = peak_membrane * PA_TO_MMHG;
    s.mean_membrane_pressure_pa = mean_membrane;
    s.mean_membrane_pressure_mmhg = mean_membrane * PA_TO_MMHG;
    s.peak_pressure_pa = peak_p;
    s.peak_pressure_mmhg = peak_p * PA_TO_MMHG;
    s.membrane_artifacts_total = artifacts_total;
    s.total_drained_ml = drained_ml;
    s.injected_ml = injected;
    s.mass_balance = mass_balance;
    *out = s;
}

uint64_t orc_metrics_wall_count(const orc_metrics* m) { return m->wall_count; }

void orc_metrics_get_masks(const orc_metrics* m, uint8_t* is_wall, uint8_t* washed) {
    if (is_wall) std::memcpy(is_wall, m->is_wall.data(), m->is_wall.size());
    if (washed) std::memcpy(washed, m->washed.data(), m->washed.size());
}

void orc_membrane_stats(const double* values, size_t n, double cap, double* mean, double* peak,
                        uint64_t* artifacts) {
    std::vector<double> v(values, values + n);
    membrane_stats(v, cap, *mean, *peak, *artifacts);
}

void orc_hash_jitter(uint64_t key, double out[3]) { to(hash_jitter(key), out); }


void orc_render_slice_dims(const orc_solver* s, const orc_slice_plane* p, uint32_t target_px, uint32_t* w,
                           uint32_t* h) {
    double mn[3], mx[3], wm, hm;
    slice_dims(*s, *p, target_px, *w, *h, mn, mx, wm, hm);
}

void orc_render_slice(const orc_solver* s, const orc_slice_plane* pl, uint32_t target_px, double vmax,
                      uint8_t* rgb) {  // render.rs:139-236
    const orc_slice_plane& p = *pl;
    double mn[3], mx[3], wm, hm;
    uint32_t w, h;
    slice_dims(*s, p, target_px, w, h, mn, mx, wm, hm);
    Rgb8 im{w, h, rgb};
    for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x < w; ++x) im.set(x, y, RC_BG);
    const double oa_lo = mn[p.oax];
    const double oa_span = fmax_(mx[p.oax] - mn[p.oax], 1e-9);
    const int PROJ_SAMPLES = 96;
    for (uint32_t py = 0; py < h; ++py)
        for (uint32_t px = 0; px < w; ++px) {  // in_plane_world, render.rs:319-338
            double wx = mn[p.hax] + ((double)px + 0.5) / (double)w * wm;
            double wy = p.flip_v ? mx[p.vax] - ((double)py + 0.5) / (double)h * hm
                                 : mn[p.vax] + ((double)py + 0.5) / (double)h * hm;
            double c[3] = {0, 0, 0};
            c[p.hax] = wx;
            c[p.vax] = wy;
            bool interior = false;
            if (p.project) {
                for (int q = 0; q < PROJ_SAMPLES && !interior; ++q) {
                    c[p.oax] = oa_lo + ((double)q + 0.5) / (double)PROJ_SAMPLES * oa_span;
                    interior = s->solid.sample(v3(c[0], c[1], c[2])) < 0.0;
                }
            } else {
                c[p.oax] = p.slice;
                interior = s->solid.sample(v3(c[0], c[1], c[2])) < 0.0;
            }
            im.set(px, py, interior ? RC_INTERIOR : RC_WALL);
        }
    auto to_px = [&](V3 a, int64_t& cx, int64_t& cy) {
        double fx = (comp(a, p.hax) - mn[p.hax]) / wm * (double)w;
        double fy = p.flip_v ? (mx[p.vax] - comp(a, p.vax)) / hm * (double)h
                             : (comp(a, p.vax) - mn[p.vax]) / hm * (double)h;
        cx = as_i64(fx);
        cy = as_i64(fy);
    };
    if (p.amber) {  // draw_amber_pool, render.rs:238-308
        const double longest = (double)(w > h ? w : h);
        const int64_t r = as_i64(fmax_(std::round(longest / 80.0), 3.0));
        const double PEAK = 0.22;
        const double rr = (double)(r * r);
        std::vector<double> cov((size_t)w * h, 0.0);
        for (V3 q : s->pos) {
            if (std::fabs(comp(q, p.oax) - p.slice) > p.slab) continue;
            int64_t cx, cy;
            to_px(q, cx, cy);
            for (int64_t dy = -r; dy <= r; ++dy)
                for (int64_t dx = -r; dx <= r; ++dx) {
                    double d2 = (double)(dx * dx + dy * dy);
                    if (d2 > rr) continue;
                    int64_t x = cx + dx, y = cy + dy;
                    if (x < 0 || y < 0 || (uint64_t)x >= w || (uint64_t)y >= h) continue;
                    double a = PEAK * (1.0 - d2 / rr);
                    size_t idx = (size_t)y * w + (size_t)x;
                    cov[idx] += (1.0 - cov[idx]) * a;
                }
        }
        for (uint32_t py = 0; py < h; ++py)
            for (uint32_t px = 0; px < w; ++px) {
                double c = clamp01(cov[(size_t)py * w + px]);
                if (c <= 1.0 / 255.0) continue;
                uint8_t amber[3], out[3];
                const uint8_t* bg = rgb + 3 * ((size_t)py * w + px);
                for (int k = 0; k < 3; ++k) amber[k] = r_lerp(RC_FILM[k], RC_DEEP[k], c);
                for (int k = 0; k < 3; ++k) out[k] = r_lerp(bg[k], amber[k], c);
                im.set(px, py, out);
            }
    } else {
        double vm = vmax > 0.0 ? vmax : fmax_(s->max_speed(), 1e-6);
        for (size_t i = 0; i < s->pos.size(); ++i) {
            V3 q = s->pos[i];
            if (std::fabs(comp(q, p.oax) - p.slice) > p.slab) continue;
            int64_t cx, cy;
            to_px(q, cx, cy);
            uint8_t col[3];
            r_speed(clamp01(length(s->vel[i]) / vm), col);
            r_disk(im, cx, cy, 2, col);
        }
    }
    V3 tip = s->needle.tip;  // render.rs:224-231
    V3 back = tip - s->needle.axis * 0.012;
    int64_t ax, ay, bx, by;
    to_px(back, ax, ay);
    to_px(tip, bx, by);
    r_line(im, ax, ay, bx, by, RC_NEEDLE);
    r_disk(im, bx, by, 3, RC_NEEDLE);
}

void orc_render_timeseries(const orc_frame_metrics* frames, size_t n, uint32_t width, uint32_t height,
                           uint8_t* rgb) {  // render.rs:351-406
    Rgb8 im{width, height, rgb};
    const uint8_t bgc[3] = {250, 250, 252};
    for (uint32_t y = 0; y < height; ++y)
        for (uint32_t x = 0; x < width; ++x) im.set(x, y, bgc);
    const int64_t x0 = 8, x1 = (int64_t)width - 8, y0 = 8, y1 = (int64_t)height - 8;
    const uint8_t grid[3] = {220, 220, 226}, axis[3] = {120, 120, 130};
    for (int64_t g = 0; g <= 4; ++g) {
        int64_t y = y1 - (y1 - y0) * g / 4;
        r_line(im, x0, y, x1, y, grid);
    }
    r_line(im, x0, y0, x0, y1, axis);
    r_line(im, x0, y1, x1, y1, axis);
    if (n < 2) return;
    double peak_p = 0.0;
    for (size_t i = 0; i < n; ++i) peak_p = fmax_(peak_p, frames[i].peak_wall_pressure_pa);
    peak_p = fmax_(peak_p, 1e-9);
    auto map = [&](size_t i, double val, int64_t& px, int64_t& py) {
        double fx = (double)x0 + (double)(x1 - x0) * (double)i / (double)(n - 1);
        double v = clamp01(val);
        double fy = (double)y1 - (double)(y1 - y0) * v;
        px = as_i64(fx);
        py = as_i64(fy);
    };
    const uint8_t cols[3][3] = {{40, 90, 220}, {30, 160, 60}, {210, 60, 50}};
    for (int sidx = 0; sidx < 3; ++sidx) {
        auto f = [&](const orc_frame_metrics& m) {
            return sidx == 0 ? m.fill_fraction : (sidx == 1 ? m.wall_coverage : m.peak_wall_pressure_pa / peak_p);
        };
        for (size_t i = 1; i < n; ++i) {
            int64_t xa, ya, xb, yb;
            map(i - 1, f(frames[i - 1]), xa, ya);
            map(i, f(frames[i]), xb, yb);
            r_line(im, xa, ya, xb, yb, cols[sidx]);
        }
    }
}
}  // extern "C"
