// Grid-side kernels: static cavity mask and base labels (solver.rs:184-222,
// 342-361), velocity extrapolation (solver.rs:608-647, 960-1009) and the
// face max-reduction behind cfl_dt (grid.rs:202-206).
#pragma once
#include "common.cuh"
#include "particles.cuh"

namespace sdr {

// Sdf::sample (sdf.rs:134-166) in f64 with the reference's operation order.
__device__ __forceinline__ void clamp_base_d(double g, int n, int& i, double& f) {
    if (g <= 0.0) {
        i = 0;
        f = 0.0;
    } else if (g >= (double)(n - 1)) {
        i = n - 2;
        f = 1.0;
    } else {
        double fl = floor(g);
        i = (int)fl;
        f = dsub(g, fl);
    }
}

struct SdfD {
    int nx, ny, nz;
    double dx, ox, oy, oz;
    const double* data;
};

__device__ __forceinline__ double sdf_sample_d(const SdfD& s, double px, double py, double pz) {
    double lx = ddiv(dsub(px, s.ox), s.dx), ly = ddiv(dsub(py, s.oy), s.dx),
           lz = ddiv(dsub(pz, s.oz), s.dx);
    int i, j, k;
    double fx, fy, fz;
    clamp_base_d(lx, s.nx, i, fx);
    clamp_base_d(ly, s.ny, j, fy);
    clamp_base_d(lz, s.nz, k, fz);
    auto at = [&](int a, int b, int c) { return s.data[((size_t)c * s.ny + b) * s.nx + a]; };
    double gx = dsub(1.0, fx), gy = dsub(1.0, fy), gz = dsub(1.0, fz);
    double c00 = dadd(dmul(at(i, j, k), gx), dmul(at(i + 1, j, k), fx));
    double c10 = dadd(dmul(at(i, j + 1, k), gx), dmul(at(i + 1, j + 1, k), fx));
    double c01 = dadd(dmul(at(i, j, k + 1), gx), dmul(at(i + 1, j, k + 1), fx));
    double c11 = dadd(dmul(at(i, j + 1, k + 1), gx), dmul(at(i + 1, j + 1, k + 1), fx));
    double c0 = dadd(dmul(c00, gy), dmul(c10, fy));
    double c1 = dadd(dmul(c01, gy), dmul(c11, fy));
    return dadd(dmul(c0, gz), dmul(c1, fz));
}

// cavity_mask (solver.rs:194-199) and the static half of classify
// (solver.rs:344-361): outlet cells are Air, non-cavity Solid, the rest Air.
__device__ __forceinline__ void k_cavity_and_base_body(VB vb_, Grid g, SdfD s, int has_outlet, Aabb outlet,
                                  uint8_t* __restrict__ cavity, uint8_t* __restrict__ base,
                                  int recompute_cavity) {
    size_t c = (size_t)vb_.bid * blockDim.x + threadIdx.x;
    size_t n = (size_t)g.nx * g.ny * g.nz;
    if (c >= n) return;
    int i = c % g.nx, j = (c / g.nx) % g.ny, k = c / ((size_t)g.nx * g.ny);
    double cx = dadd(g.ox, dmul((double)i + 0.5, g.dx));
    double cy = dadd(g.oy, dmul((double)j + 0.5, g.dx));
    double cz = dadd(g.oz, dmul((double)k + 0.5, g.dx));
    uint8_t cav;
    if (recompute_cavity) {
        cav = sdf_sample_d(s, cx, cy, cz) < 0.0 ? 1 : 0;
        cavity[c] = cav;
    } else {
        cav = cavity[c];
    }
    bool out = has_outlet && aabb_contains(outlet, cx, cy, cz);
    base[c] = out ? AIR : (!cav ? SOLID : AIR);
}
__global__ void k_cavity_and_base(Grid g, SdfD s, int has_outlet, Aabb outlet,
                                  uint8_t* __restrict__ cavity, uint8_t* __restrict__ base,
                                  int recompute_cavity) { k_cavity_and_base_body(VB{blockIdx.x, gridDim.x}, g, s, has_outlet, outlet, cavity, base, recompute_cavity); }

// Validity for extrapolation: the face borders a Fluid cell (solver.rs:612-642).
__device__ __forceinline__ void k_extrap_valid_body(VB vb_, Grid g, const uint8_t* __restrict__ cells, uint8_t* __restrict__ ku,
                               uint8_t* __restrict__ kv, uint8_t* __restrict__ kw) {
    int i, j, k;
    if (!node_of(g, (size_t)vb_.bid * blockDim.x + threadIdx.x, i, j, k)) return;
    auto fl = [&](int a, int b, int c) {
        return cells[((size_t)c * g.ny + b) * g.nx + a] == FLUID;
    };
    if (j < g.ny && k < g.nz)
        ku[((size_t)k * g.ny + j) * (g.nx + 1) + i] = (i > 0 && fl(i - 1, j, k)) || (i < g.nx && fl(i, j, k));
    if (i < g.nx && k < g.nz)
        kv[((size_t)k * (g.ny + 1) + j) * g.nx + i] = (j > 0 && fl(i, j - 1, k)) || (j < g.ny && fl(i, j, k));
    if (i < g.nx && j < g.ny)
        kw[((size_t)k * g.ny + j) * g.nx + i] = (k > 0 && fl(i, j, k - 1)) || (k < g.nz && fl(i, j, k));
}
__global__ void k_extrap_valid(Grid g, const uint8_t* __restrict__ cells, uint8_t* __restrict__ ku,
                               uint8_t* __restrict__ kv, uint8_t* __restrict__ kw) { k_extrap_valid_body(VB{blockIdx.x, gridDim.x}, g, cells, ku, kv, kw); }

// One snapshot sweep of extrapolate (solver.rs:964-1007) on one component,
// in place. kn holds 0 for unknown, 1 for known from the start and s + 2 for
// a face that became known in sweep s; sweep s reads only faces known before
// it, whose values no longer change, so every face sees the snapshot the
// reference's copy-then-update sweep gives it. Unknown entries take the mean
// of their known neighbours, summed in the order -x,+x,-y,+y,-z,+z; everything
// else is left as it is (the reference copies it unchanged).
__device__ __forceinline__ void extrap_one(float* __restrict__ f, uint8_t* __restrict__ kn, int sweep, int nx,
                                           int ny, int nz, int i, int j, int k) {
    const size_t c = ((size_t)k * ny + j) * nx + i;
    if (kn[c]) return;
    const int before = sweep + 1;  // kn in [1, before]: known before this sweep
    auto known = [&](size_t q) {
        const int v = kn[q];
        return v != 0 && v <= before;
    };
    float sum = 0.0f;
    int cnt = 0;
    const size_t sy = nx, sz = (size_t)nx * ny;
    if (i > 0 && known(c - 1)) { sum += f[c - 1]; ++cnt; }
    if (i + 1 < nx && known(c + 1)) { sum += f[c + 1]; ++cnt; }
    if (j > 0 && known(c - sy)) { sum += f[c - sy]; ++cnt; }
    if (j + 1 < ny && known(c + sy)) { sum += f[c + sy]; ++cnt; }
    if (k > 0 && known(c - sz)) { sum += f[c - sz]; ++cnt; }
    if (k + 1 < nz && known(c + sz)) { sum += f[c + sz]; ++cnt; }
    if (cnt > 0) {
        f[c] = sum / (float)cnt;
        kn[c] = (uint8_t)(sweep + 2);
    }
}

struct ExtrapArgs {
    Grid g;
    float* u;
    float* v;
    float* w;
    uint8_t* ku;
    uint8_t* kv;
    uint8_t* kw;
    int sweep;              // 0..3
    unsigned int* maxbits;  // optional: |u|,|v|,|w| maxima (last sweep)
};

__device__ __forceinline__ void k_extrap_body(VB vb_, ExtrapArgs a) {
    const Grid& g = a.g;
    int i, j, k;
    float mu = 0.f, mv = 0.f, mw = 0.f;
    if (node_of(g, (size_t)vb_.bid * blockDim.x + threadIdx.x, i, j, k)) {
        if (j < g.ny && k < g.nz) {
            extrap_one(a.u, a.ku, a.sweep, g.nx + 1, g.ny, g.nz, i, j, k);
            if (a.maxbits) mu = fabsf(a.u[((size_t)k * g.ny + j) * (g.nx + 1) + i]);
        }
        if (i < g.nx && k < g.nz) {
            extrap_one(a.v, a.kv, a.sweep, g.nx, g.ny + 1, g.nz, i, j, k);
            if (a.maxbits) mv = fabsf(a.v[((size_t)k * (g.ny + 1) + j) * g.nx + i]);
        }
        if (i < g.nx && j < g.ny) {
            extrap_one(a.w, a.kw, a.sweep, g.nx, g.ny, g.nz + 1, i, j, k);
            if (a.maxbits) mw = fabsf(a.w[((size_t)k * g.ny + j) * g.nx + i]);
        }
    }
    if (a.maxbits) {
        // Non-negative floats order like their bit patterns: exact max via atomicMax.
        for (int o = 16; o > 0; o >>= 1) {
            mu = fmaxf(mu, __shfl_xor_sync(0xffffffffu, mu, o));
            mv = fmaxf(mv, __shfl_xor_sync(0xffffffffu, mv, o));
            mw = fmaxf(mw, __shfl_xor_sync(0xffffffffu, mw, o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMax(&a.maxbits[0], __float_as_uint(mu));
            atomicMax(&a.maxbits[1], __float_as_uint(mv));
            atomicMax(&a.maxbits[2], __float_as_uint(mw));
        }
    }
}
__global__ void __launch_bounds__(256) k_extrap(ExtrapArgs a) { k_extrap_body(VB{blockIdx.x, gridDim.x}, a); }

// Face maxima alone (used when extrapolation did not run, e.g. phase mode).
__device__ __forceinline__ void k_face_max_body(VB vb_, const float* __restrict__ f, size_t n, unsigned int* __restrict__ out) {
    float m = 0.f;
    for (size_t q = (size_t)vb_.bid * blockDim.x + threadIdx.x; q < n; q += (size_t)vb_.nb * blockDim.x)
        m = fmaxf(m, fabsf(f[q]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}
__global__ void k_face_max(const float* __restrict__ f, size_t n, unsigned int* __restrict__ out) { k_face_max_body(VB{blockIdx.x, gridDim.x}, f, n, out); }

}  // namespace sdr
