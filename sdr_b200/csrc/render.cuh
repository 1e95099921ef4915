// Preview rendering (src/render.rs:139-308) on the device: the cavity
// cross-section or silhouette from the f64 SDF, then the fluid as
// speed-coloured dots or as the translucent amber pool. Pixels equal the
// reference's, which draws sequentially:
//  * dots: a later particle overwrites an earlier one, so each pixel takes the
//    colour of the highest-index particle whose disk covers it (atomicMax on
//    index + 1, then one colouring pass);
//  * amber: the coverage update cov += (1 - cov) * a is order-dependent in
//    f64, so particles are binned by image tile in index order (the stable
//    counting sort of the particle pipeline) and each pixel merges the nine
//    neighbouring tiles' lists in index order, applying exactly the
//    reference's sequence of updates.
// The needle overlay is drawn on the host afterwards (a few dozen pixels).
#pragma once
#include "grid.cuh"

namespace sdr {

struct RenderView {
    int hax, vax, oax, flip_v, project, amber;
    double slice, slab;
    double mn[3], mx[3];
    double wm, hm;
    uint32_t w, h;
};

__device__ __forceinline__ double rv_comp(double x, double y, double z, int a) {
    return a == 0 ? x : (a == 1 ? y : z);
}

__device__ __forceinline__ long long rv_as_i64(double f) {  // Rust `as i64`: truncate, saturate, NaN -> 0
    if (isnan(f)) return 0;
    if (f >= 9223372036854775807.0) return 9223372036854775807LL;
    if (f <= -9223372036854775808.0) return (-9223372036854775807LL - 1);
    return (long long)f;
}

__device__ __forceinline__ uint8_t rv_as_u8(double f) {
    if (isnan(f) || f <= 0.0) return 0;
    if (f >= 255.0) return 255;
    return (uint8_t)f;
}

__device__ __forceinline__ double rv_clamp01(double t) { return t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t); }

// to_px (render.rs:181-191)
__device__ __forceinline__ void rv_to_px(const RenderView& v, float4 p, long long& cx, long long& cy) {
    const double a = rv_comp(p.x, p.y, p.z, v.hax), b = rv_comp(p.x, p.y, p.z, v.vax);
    const double fx = dmul(ddiv(dsub(a, v.mn[v.hax]), v.wm), (double)v.w);
    const double fy = v.flip_v ? dmul(ddiv(dsub(v.mx[v.vax], b), v.hm), (double)v.h)
                               : dmul(ddiv(dsub(b, v.mn[v.vax]), v.hm), (double)v.h);
    cx = rv_as_i64(fx);
    cy = rv_as_i64(fy);
}

__device__ __forceinline__ bool rv_in_slab(const RenderView& v, float4 p) {
    return !(fabs(dsub(rv_comp(p.x, p.y, p.z, v.oax), v.slice)) > v.slab);
}

// Background (render.rs:159-178): interior where the SDF is negative on the
// plane, or at any of 96 depths for a projection.
__global__ void k_render_bg(RenderView v, SdfD s, uint8_t* __restrict__ rgb) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (size_t)v.w * v.h) return;
    const uint32_t px = (uint32_t)(q % v.w), py = (uint32_t)(q / v.w);
    // in_plane_world (render.rs:319-338)
    const double wx = dadd(v.mn[v.hax], dmul(ddiv((double)px + 0.5, (double)v.w), v.wm));
    const double fyv = dmul(ddiv((double)py + 0.5, (double)v.h), v.hm);
    const double wy = v.flip_v ? dsub(v.mx[v.vax], fyv) : dadd(v.mn[v.vax], fyv);
    double c[3] = {0.0, 0.0, 0.0};
    c[v.hax] = wx;
    c[v.vax] = wy;
    bool interior = false;
    if (v.project) {
        const double lo = v.mn[v.oax], span = fmax(dsub(v.mx[v.oax], v.mn[v.oax]), 1e-9);
        for (int k = 0; k < 96 && !interior; ++k) {
            c[v.oax] = dadd(lo, dmul(ddiv((double)k + 0.5, 96.0), span));
            interior = sdf_sample_d(s, c[0], c[1], c[2]) < 0.0;
        }
    } else {
        c[v.oax] = v.slice;
        interior = sdf_sample_d(s, c[0], c[1], c[2]) < 0.0;
    }
    uint8_t* o = rgb + 3 * q;
    if (interior) {
        o[0] = 232; o[1] = 236; o[2] = 244;
    } else {
        o[0] = 44; o[1] = 44; o[2] = 54;
    }
}

// Peak particle speed (solver.rs:884-890) as the bit pattern of a
// non-negative double, which orders like the value.
__global__ void k_render_max_speed(const float4* __restrict__ vel, uint32_t n, unsigned long long* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double m = 0.0;
    if (i < n) {
        const float4 u = vel[i];
        m = __dsqrt_rn(dadd(dadd(dmul(u.x, u.x), dmul(u.y, u.y)), dmul(u.z, u.z)));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// Speed dots (render.rs:201-221): radius-2 disks; the highest index wins.
__global__ void k_render_dots_mark(RenderView v, const float4* __restrict__ pos, uint32_t n,
                                   uint32_t* __restrict__ owner) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i];
    if (!rv_in_slab(v, p)) return;
    long long cx, cy;
    rv_to_px(v, p, cx, cy);
    for (int dy = -2; dy <= 2; ++dy)
        for (int dx = -2; dx <= 2; ++dx) {
            if (dx * dx + dy * dy > 4) continue;
            const long long x = cx + dx, y = cy + dy;
            if (x < 0 || y < 0 || x >= (long long)v.w || y >= (long long)v.h) continue;
            atomicMax(owner + (size_t)y * v.w + x, i + 1);
        }
}

// speed_color (render.rs:417-428) of the winning particle.
__global__ void k_render_dots_color(RenderView v, const float4* __restrict__ vel, const uint32_t* __restrict__ owner,
                                    const unsigned long long* __restrict__ peak_bits, double vmax,
                                    uint8_t* __restrict__ rgb) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (size_t)v.w * v.h) return;
    const uint32_t o = owner[q];
    if (!o) return;
    const double vm = vmax > 0.0 ? vmax : fmax(__longlong_as_double((long long)*peak_bits), 1e-6);
    const float4 u = vel[o - 1];
    const double sp = __dsqrt_rn(dadd(dadd(dmul(u.x, u.x), dmul(u.y, u.y)), dmul(u.z, u.z)));
    const double t = rv_clamp01(rv_clamp01(ddiv(sp, vm)));
    double r, g, b;
    if (t < 0.5) {
        const double uu = ddiv(t, 0.5);
        r = 0.0; g = uu; b = dsub(1.0, uu);
    } else {
        const double uu = ddiv(dsub(t, 0.5), 0.5);
        r = uu; g = dsub(1.0, uu); b = 0.0;
    }
    uint8_t* c = rgb + 3 * q;
    c[0] = rv_as_u8(dmul(r, 255.0));
    c[1] = rv_as_u8(dmul(g, 255.0));
    c[2] = rv_as_u8(dmul(b, 255.0));
}

// Amber pool, binning: the tile (side T = splat radius) of each particle's
// centre pixel on a grid with one tile of margin; particles outside it (or
// the slab) go to the last bin, which no pixel reads.
__global__ void k_render_amber_keys(RenderView v, const float4* __restrict__ pos, uint32_t n, int T, int ntx,
                                    int nty, uint32_t* __restrict__ key, int2* __restrict__ cxy,
                                    uint32_t* __restrict__ hist) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t dump = (uint32_t)(ntx + 2) * (uint32_t)(nty + 2);
    const float4 p = pos[i];
    uint32_t k = dump;
    if (rv_in_slab(v, p)) {
        long long cx, cy;
        rv_to_px(v, p, cx, cy);
        const long long tx = (cx >= 0 ? cx / T : -((-cx + T - 1) / T)) + 1;
        const long long ty = (cy >= 0 ? cy / T : -((-cy + T - 1) / T)) + 1;
        if (tx >= 0 && ty >= 0 && tx <= ntx + 1 && ty <= nty + 1) {
            k = (uint32_t)(ty * (ntx + 2) + tx);
            cxy[i] = make_int2((int)cx, (int)cy);
        }
    }
    key[i] = k;
    atomicAdd(hist + k, 1u);
}

__device__ __forceinline__ uint8_t rv_lerp(uint8_t a, uint8_t b, double t) {  // lerp_u8, render.rs:311-316
    t = rv_clamp01(t);
    double x = round(dadd(dmul((double)a, dsub(1.0, t)), dmul((double)b, t)));
    x = x < 0.0 ? 0.0 : (x > 255.0 ? 255.0 : x);
    return (uint8_t)x;
}

// Amber pool, compositing (render.rs:261-307): every pixel replays, in
// particle order, the splats of the particles binned in its 3x3 tiles.
__global__ void k_render_amber_pixels(RenderView v, int r, int T, int ntx, const uint32_t* __restrict__ start,
                                      const uint32_t* __restrict__ perm, const int2* __restrict__ cxy,
                                      uint8_t* __restrict__ rgb) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (size_t)v.w * v.h) return;
    const int x = (int)(q % v.w), y = (int)(q / v.w);
    const int tx = x / T + 1, ty = y / T + 1;
    uint32_t cur[9], end[9];
    for (int b = 0; b < 9; ++b) {
        const uint32_t bin = (uint32_t)(ty + b / 3 - 1) * (uint32_t)(ntx + 2) + (uint32_t)(tx + b % 3 - 1);
        cur[b] = start[bin];
        end[b] = start[bin + 1];
    }
    const double rr = (double)((long long)r * r);
    double cov = 0.0;
    for (;;) {
        uint32_t best = 0xFFFFFFFFu;
        int bb = -1;
        for (int b = 0; b < 9; ++b)
            if (cur[b] < end[b]) {
                const uint32_t pi = perm[cur[b]];
                if (pi < best) {
                    best = pi;
                    bb = b;
                }
            }
        if (bb < 0) break;
        ++cur[bb];
        const int2 c = cxy[best];
        const long long dx = (long long)x - c.x, dy = (long long)y - c.y;
        if (dx < -r || dx > r || dy < -r || dy > r) continue;
        const double d2 = (double)(dx * dx + dy * dy);
        if (d2 > rr) continue;
        const double a = dmul(0.22, dsub(1.0, ddiv(d2, rr)));
        cov = dadd(cov, dmul(dsub(1.0, cov), a));
    }
    const double cc = rv_clamp01(cov);
    if (cc <= 1.0 / 255.0) return;
    uint8_t* o = rgb + 3 * q;
    const uint8_t film[3] = {242, 178, 92}, deep[3] = {150, 78, 18};
    for (int k = 0; k < 3; ++k) {
        const uint8_t amber = rv_lerp(film[k], deep[k], cc);
        o[k] = rv_lerp(o[k], amber, cc);
    }
}

}  // namespace sdr
