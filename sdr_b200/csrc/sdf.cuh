// SDF builders on the device.
//  * k_sdf_mesh: Sdf::from_mesh_in_bounds (sdf.rs:53-86) — per node, min
//    closest-point distance (Ericson, sdf.rs:209-254) and the summed van
//    Oosterom–Strackee solid angle (sdf.rs:259-272) over all triangles, sign
//    from winding > 1/2 (sdf.rs:187-205). Triangles stream through shared
//    memory in tiles moved by the bulk-copy engine (cp.async.bulk, one
//    transaction per tile into the CTA's own shared memory, no multicast),
//    double-buffered behind an mbarrier with a bounded wait.
//  * k_sdf_sinus: Sdf::from_fn(SinusParams::implicit) (sinus.rs:89-119).
// All arithmetic is f64 without contraction, in the reference's order.
#pragma once
#include "common.cuh"

namespace sdr {

struct D3 {
    double x, y, z;
};
__device__ __forceinline__ D3 d3(double x, double y, double z) { return D3{x, y, z}; }
__device__ __forceinline__ D3 sub3(D3 a, D3 b) { return d3(dsub(a.x, b.x), dsub(a.y, b.y), dsub(a.z, b.z)); }
__device__ __forceinline__ D3 add3(D3 a, D3 b) { return d3(dadd(a.x, b.x), dadd(a.y, b.y), dadd(a.z, b.z)); }
__device__ __forceinline__ D3 mul3(D3 a, double s) { return d3(dmul(a.x, s), dmul(a.y, s), dmul(a.z, s)); }
__device__ __forceinline__ double dot3(D3 a, D3 b) { return dadd(dadd(dmul(a.x, b.x), dmul(a.y, b.y)), dmul(a.z, b.z)); }
__device__ __forceinline__ D3 cross3(D3 a, D3 b) {
    return d3(dsub(dmul(a.y, b.z), dmul(a.z, b.y)), dsub(dmul(a.z, b.x), dmul(a.x, b.z)),
              dsub(dmul(a.x, b.y), dmul(a.y, b.x)));
}

__device__ __forceinline__ double tri_dist_sq(D3 p, D3 a, D3 b, D3 c) {  // sdf.rs:209-254
    D3 ab = sub3(b, a), ac = sub3(c, a), ap = sub3(p, a);
    double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) return dot3(ap, ap);
    D3 bp = sub3(p, b);
    double d3_ = dot3(ab, bp), d4 = dot3(ac, bp);
    if (d3_ >= 0.0 && d4 <= d3_) return dot3(bp, bp);
    double vc = dsub(dmul(d1, d4), dmul(d3_, d2));
    if (vc <= 0.0 && d1 >= 0.0 && d3_ <= 0.0) {
        double v = ddiv(d1, dsub(d1, d3_));
        D3 e = sub3(p, add3(a, mul3(ab, v)));
        return dot3(e, e);
    }
    D3 cp = sub3(p, c);
    double d5 = dot3(ab, cp), d6 = dot3(ac, cp);
    if (d6 >= 0.0 && d5 <= d6) return dot3(cp, cp);
    double vb = dsub(dmul(d5, d2), dmul(d1, d6));
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        double w = ddiv(d2, dsub(d2, d6));
        D3 e = sub3(p, add3(a, mul3(ac, w)));
        return dot3(e, e);
    }
    double va = dsub(dmul(d3_, d6), dmul(d5, d4));
    if (va <= 0.0 && dsub(d4, d3_) >= 0.0 && dsub(d5, d6) >= 0.0) {
        double w = ddiv(dsub(d4, d3_), dadd(dsub(d4, d3_), dsub(d5, d6)));
        D3 e = sub3(p, add3(b, mul3(sub3(c, b), w)));
        return dot3(e, e);
    }
    double denom = ddiv(1.0, dadd(dadd(va, vb), vc));
    double v = dmul(vb, denom), w = dmul(vc, denom);
    D3 e = sub3(p, add3(add3(a, mul3(ab, v)), mul3(ac, w)));
    return dot3(e, e);
}

__device__ __forceinline__ double solid_angle(D3 p, D3 a, D3 b, D3 c) {  // sdf.rs:259-272
    D3 av = sub3(a, p), bv = sub3(b, p), cv = sub3(c, p);
    double la = __dsqrt_rn(dot3(av, av)), lb = __dsqrt_rn(dot3(bv, bv)), lc = __dsqrt_rn(dot3(cv, cv));
    if (la < 1e-12 || lb < 1e-12 || lc < 1e-12) return 0.0;
    double num = dot3(av, cross3(bv, cv));
    double den = dadd(dadd(dadd(dmul(dmul(la, lb), lc), dmul(dot3(av, bv), lc)), dmul(dot3(bv, cv), la)),
                      dmul(dot3(cv, av), lb));
    return dmul(2.0, atan2(num, den));
}

constexpr int kSdfBS = 128;
constexpr int kSdfTile = 128;  // triangles per stage (9216 bytes)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// Bounded wait on an mbarrier phase: gives up after about one second of SM
// clock (2^31 cycles, 1.1 s at 1965 MHz) and returns false.
constexpr long long kWaitCycles = 1ll << 31;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const long long t0 = clock64();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > kWaitCycles) return false;
    }
}

// k_sdf_mesh's test hook: the tile whose bulk copy is not issued (so its
// staging wait runs out); kNoSkip in normal use.
constexpr uint32_t kNoSkip = 0xFFFFFFFFu;

// tris: padded to a whole number of tiles (9 f64 per triangle, 16-byte aligned).
__global__ void __launch_bounds__(kSdfBS) k_sdf_mesh(const double* __restrict__ tris, uint32_t ntri,
                                                     uint32_t ntiles, double ox, double oy, double oz,
                                                     double dx, int nx, int ny, int nz,
                                                     double* __restrict__ out, uint32_t* __restrict__ err,
                                                     uint32_t skip_tile = kNoSkip) {
    __shared__ __align__(128) double st[2][kSdfTile * 9];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ int fail;
    size_t node = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    size_t nn = (size_t)nx * ny * nz;
    int i = node % nx, j = (node / nx) % ny, k = node / ((size_t)nx * ny);
    D3 p = d3(dadd(ox, dmul((double)i, dx)), dadd(oy, dmul((double)j, dx)), dadd(oz, dmul((double)k, dx)));
    if (threadIdx.x == 0) {
        fail = 0;
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const uint32_t bytes = kSdfTile * 9 * sizeof(double);
    uint32_t issued = 0;  // thread 0 only
    if (threadIdx.x == 0 && ntiles > 0) {
        if (skip_tile != 0) bulk_load(st[0], tris, bytes, &bar[0]);
        issued = 1;
    }
    double min_d2 = INFINITY, wind = 0.0;
    uint32_t t = 0;
    for (; t < ntiles; ++t) {
        int b = t & 1;
        if (threadIdx.x == 0 && t + 1 < ntiles) {
            if (skip_tile != t + 1) bulk_load(st[b ^ 1], tris + (size_t)(t + 1) * kSdfTile * 9, bytes, &bar[b ^ 1]);
            issued = t + 2;
        }
        if (!mbar_wait(&bar[b], (t >> 1) & 1)) fail = 1;
        __syncthreads();
        if (fail) break;
        uint32_t cnt = min((uint32_t)kSdfTile, ntri - t * kSdfTile);
        const double* s = st[b];
        for (uint32_t q = 0; q < cnt; ++q) {
            D3 a = d3(s[9 * q], s[9 * q + 1], s[9 * q + 2]);
            D3 bb = d3(s[9 * q + 3], s[9 * q + 4], s[9 * q + 5]);
            D3 c = d3(s[9 * q + 6], s[9 * q + 7], s[9 * q + 8]);
            double d2 = tri_dist_sq(p, a, bb, c);
            if (d2 < min_d2) min_d2 = d2;
            wind = dadd(wind, solid_angle(p, a, bb, c));
        }
        __syncthreads();  // everyone is done with st[b] before it is refilled
    }
    if (fail) {
        // A bounded wait gave up: drain the copies still in flight (again
        // bounded) before the block's shared memory goes away, then report.
        if (threadIdx.x == 0) {
            for (uint32_t q = t; q < issued; ++q)
                if (q != skip_tile) mbar_wait(&bar[q & 1], (q >> 1) & 1);
            atomicOr(err, 1u);
        }
        return;
    }
    if (node >= nn) return;
    wind = ddiv(wind, dmul(4.0, 3.141592653589793));
    double dist = __dsqrt_rn(min_d2);
    out[node] = wind > 0.5 ? -dist : dist;
}

struct SinusD {
    double ax, ay, az, cx, cy, cz, taper, bump, sx, sz, sr, sd;
};

__device__ __forceinline__ double clampd(double x, double lo, double hi) {
    return x < lo ? lo : (x > hi ? hi : x);
}

__device__ __forceinline__ double sinus_implicit(const SinusD& s, double px, double py, double pz) {
    double qx = dsub(px, s.cx), qy = dsub(py, s.cy), qz = dsub(pz, s.cz);
    double h = dmul(dadd(ddiv(qy, s.ay), 1.0), 0.5);
    double scale = dadd(s.taper, dmul(dsub(1.0, s.taper), clampd(h, 0.0, 1.5)));
    double bump = dmul(s.bump, dadd(dmul(dmul(0.6, sin(ddiv(dmul(4.0, qx), s.ax))), cos(ddiv(dmul(3.0, qz), s.az))),
                                    dmul(0.4, sin(dadd(ddiv(dmul(5.0, qy), s.ay), 1.3)))));
    double tx = ddiv(qx, dmul(s.ax, scale)), ty = ddiv(qy, s.ay), tz = ddiv(qz, dmul(s.az, scale));
    double body = dsub(__dsqrt_rn(dadd(dadd(dmul(tx, tx), dmul(ty, ty)), dmul(tz, tz))), dadd(1.0, bump));
    body = dmul(body, fmin(fmin(s.ax, s.ay), s.az));
    double rx = dsub(px, s.sx), rz = dsub(pz, s.sz);
    double radial = dsub(__dsqrt_rn(dadd(dmul(rx, rx), dmul(rz, rz))), s.sr);
    double ytop = dsub(s.cy, dmul(0.5, s.ay));
    double ybot = dsub(dsub(s.cy, s.ay), s.sd);
    double axial = fmax(dsub(py, ytop), dsub(ybot, py));
    double socket = fmax(radial, axial);
    const double kk = 0.0015;
    double hh = clampd(dadd(0.5, ddiv(dmul(0.5, dsub(socket, body)), kk)), 0.0, 1.0);
    return dsub(dadd(dmul(socket, dsub(1.0, hh)), dmul(body, hh)), dmul(dmul(kk, hh), dsub(1.0, hh)));
}

__global__ void k_sdf_sinus(SinusD s, double ox, double oy, double oz, double dx, int nx, int ny, int nz,
                            double* __restrict__ out) {
    size_t node = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= (size_t)nx * ny * nz) return;
    int i = node % nx, j = (node / nx) % ny, k = node / ((size_t)nx * ny);
    out[node] = sinus_implicit(s, dadd(ox, dmul((double)i, dx)), dadd(oy, dmul((double)j, dx)),
                               dadd(oz, dmul((double)k, dx)));
}

}  // namespace sdr
