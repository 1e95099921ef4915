// Shared device types and helpers for the sdr B200 substep kernels.
//
// Precision contract (FP32 transfers, FP64 solve):
//  * particle state, MAC faces and SDF samples used by advection are f32;
//  * cell keys for labels/histograms, the pressure RHS, the MIC(0) factor,
//    the PCG vectors, dots and residual norms are f64, computed with explicit
//    round-to-nearest intrinsics so no FMA contraction changes the reference's
//    operation order (src/pressure.rs:123-609).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace sdr {

enum : uint8_t { SOLID = 0, FLUID = 1, AIR = 2 };

constexpr int kInvalid = -1;

// ---------------------------------------------------------------- GPU-scope ordering
__device__ __forceinline__ unsigned long long ld_acquire_gpu(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned ld_acquire_gpu_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu_u32(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned atom_add_acqrel_gpu(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

constexpr long long kGridWaitCycles = 1ll << 31;  // ~1.1 s at 1965 MHz
constexpr uint32_t kErrGridWait = 32u;            // error bit: a grid barrier gave up

// Barrier over every CTA of a cooperative launch: an arrival counter and a
// generation word (release/acquire at GPU scope). It gives up after about a
// second, or at once when another CTA already has (error word non-zero),
// sets `bit` in *err and returns false; every CTA then winds down.
__device__ inline bool grid_sync_bounded(unsigned* bar, uint32_t* err, uint32_t bit) {
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned gen = ld_acquire_gpu_u32(bar + 1);
        const unsigned arrived = atom_add_acqrel_gpu(bar, 1u) + 1u;
        if (arrived == gridDim.x) {
            bar[0] = 0u;  // ordered before the release of the next generation
            st_release_gpu_u32(bar + 1, gen + 1u);
        } else {
            const long long t0 = clock64();
            while (ld_acquire_gpu_u32(bar + 1) == gen) {
                if (*(volatile uint32_t*)err != 0u) {
                    ok = 0;
                    break;
                }
                if (clock64() - t0 > kGridWaitCycles) {
                    atomicOr(err, bit);
                    ok = 0;
                    break;
                }
            }
        }
        if (ok && *(volatile uint32_t*)err != 0u) ok = 0;
        ok_s = ok;
    }
    __syncthreads();
    return ok_s != 0;
}

// The block a kernel body runs as: its index and the block count of its
// launch. A plain launch passes (blockIdx.x, gridDim.x); a packed launch of
// many scenes passes the block's place within its own scene's share.
struct VB {
    uint32_t bid, nb;
};

// Uncontracted f64 arithmetic (the reference's Rust emits no FMA).
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

struct Aabb {
    double mn[3], mx[3];
};

// MAC grid geometry (src/grid.rs:92-100).
struct Grid {
    int nx, ny, nz;
    double dx, ox, oy, oz;
    float dxf, oxf, oyf, ozf;
};

// Node-grid SDF (src/sdf.rs:23-34), f32 copy for hot sampling.
struct Sdf {
    int nx, ny, nz;
    float dx, ox, oy, oz;
    const float* data;
};

__device__ __forceinline__ bool aabb_contains(const Aabb& b, double x, double y, double z) {
    // math.rs:249-256 (inclusive)
    return x >= b.mn[0] && x <= b.mx[0] && y >= b.mn[1] && y <= b.mx[1] && z >= b.mn[2] &&
           z <= b.mx[2];
}

// Solver::cell_of (solver.rs:897-908) in f64 on the (f32) particle position:
// the same arithmetic as the reference applied to the same stored values.
__device__ __forceinline__ int cell_of(const Grid& g, float px, float py, float pz) {
    double lx = ddiv(dsub((double)px, g.ox), g.dx);
    double ly = ddiv(dsub((double)py, g.oy), g.dx);
    double lz = ddiv(dsub((double)pz, g.oz), g.dx);
    if (!(lx >= 0.0) || !(ly >= 0.0) || !(lz >= 0.0)) return kInvalid;  // also rejects NaN
    if (lx >= (double)g.nx || ly >= (double)g.ny || lz >= (double)g.nz) return kInvalid;
    int i = (int)lx, j = (int)ly, k = (int)lz;
    return (k * g.ny + j) * g.nx + i;
}

// clamp_base of grid.rs:25-34 / sdf.rs:136-145 in f32.
__device__ __forceinline__ void clamp_base(float g, int n, int& i, float& f) {
    if (!(g > 0.0f)) {  // g <= 0 or NaN
        i = 0;
        f = 0.0f;
    } else if (g >= (float)(n - 1)) {
        i = n - 2;
        f = 1.0f;
    } else {
        float fl = floorf(g);
        i = (int)fl;
        f = g - fl;
    }
}

// trilinear_sample (grid.rs:18-47), f32, dims = node counts (x fastest).
__device__ __forceinline__ float trilerp(const float* __restrict__ a, int nx, int ny, int nz,
                                         float gx, float gy, float gz) {
    int i, j, k;
    float fx, fy, fz;
    clamp_base(gx, nx, i, fx);
    clamp_base(gy, ny, j, fy);
    clamp_base(gz, nz, k, fz);
    size_t b = ((size_t)k * ny + j) * nx + i;
    size_t sy = nx, sz = (size_t)nx * ny;
    float c00 = a[b] * (1.0f - fx) + a[b + 1] * fx;
    float c10 = a[b + sy] * (1.0f - fx) + a[b + sy + 1] * fx;
    float c01 = a[b + sz] * (1.0f - fx) + a[b + sz + 1] * fx;
    float c11 = a[b + sy + sz] * (1.0f - fx) + a[b + sy + sz + 1] * fx;
    float c0 = c00 * (1.0f - fy) + c10 * fy;
    float c1 = c01 * (1.0f - fy) + c11 * fy;
    return c0 * (1.0f - fz) + c1 * fz;
}

// Same stencil on the difference field (a - b), for the FLIP delta (solver.rs:652-673).
__device__ __forceinline__ float trilerp_diff(const float* __restrict__ a,
                                              const float* __restrict__ b, int nx, int ny, int nz,
                                              float gx, float gy, float gz) {
    int i, j, k;
    float fx, fy, fz;
    clamp_base(gx, nx, i, fx);
    clamp_base(gy, ny, j, fy);
    clamp_base(gz, nz, k, fz);
    size_t o = ((size_t)k * ny + j) * nx + i;
    size_t sy = nx, sz = (size_t)nx * ny;
#define D(q) (a[q] - b[q])
    float c00 = D(o) * (1.0f - fx) + D(o + 1) * fx;
    float c10 = D(o + sy) * (1.0f - fx) + D(o + sy + 1) * fx;
    float c01 = D(o + sz) * (1.0f - fx) + D(o + sz + 1) * fx;
    float c11 = D(o + sy + sz) * (1.0f - fx) + D(o + sy + sz + 1) * fx;
#undef D
    float c0 = c00 * (1.0f - fy) + c10 * fy;
    float c1 = c01 * (1.0f - fy) + c11 * fy;
    return c0 * (1.0f - fz) + c1 * fz;
}

struct Faces {
    const float* u;
    const float* v;
    const float* w;
};

// MacGrid::velocity_at (grid.rs:191), f32.
__device__ __forceinline__ float3 velocity_at(const Grid& g, Faces f, float px, float py,
                                              float pz) {
    float lx = (px - g.oxf) / g.dxf, ly = (py - g.oyf) / g.dxf, lz = (pz - g.ozf) / g.dxf;
    float3 r;
    r.x = trilerp(f.u, g.nx + 1, g.ny, g.nz, lx, ly - 0.5f, lz - 0.5f);
    r.y = trilerp(f.v, g.nx, g.ny + 1, g.nz, lx - 0.5f, ly, lz - 0.5f);
    r.z = trilerp(f.w, g.nx, g.ny, g.nz + 1, lx - 0.5f, ly - 0.5f, lz);
    return r;
}

// Sdf::sample (sdf.rs:134-166), f32.
__device__ __forceinline__ float sdf_sample(const Sdf& s, float px, float py, float pz) {
    float lx = (px - s.ox) / s.dx, ly = (py - s.oy) / s.dx, lz = (pz - s.oz) / s.dx;
    return trilerp(s.data, s.nx, s.ny, s.nz, lx, ly, lz);
}

// Sdf::gradient (sdf.rs:170-176), f32 central differences.
__device__ __forceinline__ float3 sdf_gradient(const Sdf& s, float px, float py, float pz) {
    float h = s.dx;
    float gx = sdf_sample(s, px + h, py, pz) - sdf_sample(s, px - h, py, pz);
    float gy = sdf_sample(s, px, py + h, pz) - sdf_sample(s, px, py - h, pz);
    float gz = sdf_sample(s, px, py, pz + h) - sdf_sample(s, px, py, pz - h);
    float d = 2.0f * h;
    return make_float3(gx / d, gy / d, gz / d);
}

// Vec3::normalize_or_zero (math.rs:73-80), f32.
__device__ __forceinline__ float3 normalize_or_zero(float3 a) {
    float len = sqrtf(a.x * a.x + a.y * a.y + a.z * a.z);
    if (len > 1e-12f) return make_float3(a.x / len, a.y / len, a.z / len);
    return make_float3(0.f, 0.f, 0.f);
}

// Solver::project_inside (solver.rs:717-732), f32; margin is half a grid cell.
__device__ __forceinline__ float3 project_inside(const Sdf& s, float margin, float3 p) {
    for (int it = 0; it < 3; ++it) {
        float phi = sdf_sample(s, p.x, p.y, p.z);
        if (phi <= -margin) break;
        float3 g = normalize_or_zero(sdf_gradient(s, p.x, p.y, p.z));
        if (sqrtf(g.x * g.x + g.y * g.y + g.z * g.z) == 0.0f) break;
        float a = phi + margin;
        p.x -= g.x * a;
        p.y -= g.y * a;
        p.z -= g.z * a;
    }
    return p;
}

// hash_jitter (solver.rs:916-930): splitmix64 finaliser -> [-0.3, 0.3)^3, f64.
__device__ __host__ __forceinline__ double jitter_mix(uint64_t k) {
    uint64_t z = k + 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return ((double)(z >> 11) / (double)(1ULL << 53) - 0.5) * 0.6;
}

// ---------------------------------------------------------------- block reductions
template <int BS>
__device__ __forceinline__ double block_max(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        v = (l < BS / 32) ? sh[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (l == 0) sh[0] = v;
    }
    __syncthreads();
    double r = sh[0];
    __syncthreads();
    return r;
}

// Deterministic f64 block sum: fixed shuffle tree, then warps in index order.
template <int BS>
__device__ __forceinline__ double block_sum(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v = dadd(v, __shfl_xor_sync(0xffffffffu, v, o));
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        v = (l < BS / 32) ? sh[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v = dadd(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (l == 0) sh[0] = v;
    }
    __syncthreads();
    double r = sh[0];
    __syncthreads();
    return r;
}

template <int BS>
__device__ __forceinline__ uint32_t block_sum_u32(uint32_t v, uint32_t* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        v = (l < BS / 32) ? sh[l] : 0u;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (l == 0) sh[0] = v;
    }
    __syncthreads();
    uint32_t r = sh[0];
    __syncthreads();
    return r;
}

// Thread-block clusters: the hardware barrier over every thread of every CTA
// of the cluster (release/acquire at cluster scope), and the CTA's place in it.
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_size() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}

}  // namespace sdr
