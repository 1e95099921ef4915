// Naive surface nets over a node field and the mesh's signed volume
// (src/surface_nets.rs:48-221, src/mesh.rs:63-70): the parametric cavity
// volume that fill fractions are quoted against (src/scene.rs:312).
// Host code: it runs once per scene on values the device already produced.
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "sdr_gpu.h"

namespace {

struct P3 {
    double x, y, z;
};
inline P3 operator+(P3 a, P3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline P3 operator-(P3 a, P3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline P3 operator*(P3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dotp(P3 a, P3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline P3 crossp(P3 a, P3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

const int kCorner[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {1, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
const int kEdge[12][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {0, 2}, {1, 3}, {4, 6}, {5, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};

void quad(const int64_t ring[4], P3 desired, const std::vector<P3>& vs, std::vector<uint32_t>& idx) {
    for (int q = 0; q < 4; ++q)
        if (ring[q] < 0) return;
    uint32_t a = (uint32_t)ring[0], b = (uint32_t)ring[1], c = (uint32_t)ring[2], d = (uint32_t)ring[3];
    P3 nrm = crossp(vs[b] - vs[a], vs[c] - vs[a]);
    if (dotp(nrm, desired) >= 0.0)
        idx.insert(idx.end(), {a, b, c, a, c, d});
    else
        idx.insert(idx.end(), {a, c, b, a, d, c});
}

}  // namespace


extern "C" int sdr_surface_nets_volume(const double* values, const uint64_t dims[3], sdr_vec3 origin, double dx,
                                       double* volume, uint64_t* triangles) {
    if (!values || !dims || !volume || dims[0] < 2 || dims[1] < 2 || dims[2] < 2 || !(dx > 0))
        return SDR_ERR_INVALID;
    const size_t nx = dims[0], ny = dims[1], nz = dims[2];
    auto node = [&](size_t i, size_t j, size_t k) { return values[(k * ny + j) * nx + i]; };
    const size_t cx = nx - 1, cy = ny - 1, cz = nz - 1;
    std::vector<int64_t> cv(cx * cy * cz, -1);
    auto cid = [&](size_t i, size_t j, size_t k) { return (k * cy + j) * cx + i; };
    std::vector<P3> vs;
    const P3 o{origin.x, origin.y, origin.z};
    for (size_t k = 0; k < cz; ++k)
        for (size_t j = 0; j < cy; ++j)
            for (size_t i = 0; i < cx; ++i) {
                double val[8];
                for (int c = 0; c < 8; ++c) val[c] = node(i + kCorner[c][0], j + kCorner[c][1], k + kCorner[c][2]);
                P3 sum{0, 0, 0};
                int cnt = 0;
                for (int e = 0; e < 12; ++e) {
                    int a = kEdge[e][0], b = kEdge[e][1];
                    if ((val[a] < 0.0) != (val[b] < 0.0)) {
                        double t = val[a] / (val[a] - val[b]);
                        P3 pa{(double)kCorner[a][0], (double)kCorner[a][1], (double)kCorner[a][2]};
                        P3 pb{(double)kCorner[b][0], (double)kCorner[b][1], (double)kCorner[b][2]};
                        sum = sum + (pa + (pb - pa) * t);
                        ++cnt;
                    }
                }
                if (!cnt) continue;
                P3 l{sum.x / cnt, sum.y / cnt, sum.z / cnt};
                cv[cid(i, j, k)] = (int64_t)vs.size();
                vs.push_back(o + P3{((double)i + l.x) * dx, ((double)j + l.y) * dx, ((double)k + l.z) * dx});
            }
    std::vector<uint32_t> idx;
    auto get = [&](size_t i, size_t j, size_t k) { return cv[cid(i, j, k)]; };
    for (size_t k = 0; k < nz; ++k)
        for (size_t j = 0; j < ny; ++j)
            for (size_t i = 0; i < nx; ++i) {
                double v0 = node(i, j, k);
                if (i + 1 < nx && j >= 1 && k >= 1) {
                    double v1 = node(i + 1, j, k);
                    if ((v0 < 0.0) != (v1 < 0.0)) {
                        int64_t ring[4] = {get(i, j - 1, k - 1), get(i, j, k - 1), get(i, j, k), get(i, j - 1, k)};
                        quad(ring, v0 < v1 ? P3{1, 0, 0} : P3{-1, 0, 0}, vs, idx);
                    }
                }
                if (j + 1 < ny && i >= 1 && k >= 1) {
                    double v1 = node(i, j + 1, k);
                    if ((v0 < 0.0) != (v1 < 0.0)) {
                        int64_t ring[4] = {get(i - 1, j, k - 1), get(i, j, k - 1), get(i, j, k), get(i - 1, j, k)};
                        quad(ring, v0 < v1 ? P3{0, 1, 0} : P3{0, -1, 0}, vs, idx);
                    }
                }
                if (k + 1 < nz && i >= 1 && j >= 1) {
                    double v1 = node(i, j, k + 1);
                    if ((v0 < 0.0) != (v1 < 0.0)) {
                        int64_t ring[4] = {get(i - 1, j - 1, k), get(i, j - 1, k), get(i, j, k), get(i - 1, j, k)};
                        quad(ring, v0 < v1 ? P3{0, 0, 1} : P3{0, 0, -1}, vs, idx);
                    }
                }
            }
    double vol = 0.0;
    for (size_t t = 0; t + 2 < idx.size(); t += 3)
        vol += dotp(vs[idx[t]], crossp(vs[idx[t + 1]], vs[idx[t + 2]])) / 6.0;
    *volume = std::fabs(vol);
    if (triangles) *triangles = idx.size() / 3;
    return SDR_OK;
}
