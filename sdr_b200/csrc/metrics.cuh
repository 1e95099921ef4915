// Per-frame clinical metrics on the device (src/metrics.rs:119-316).
// Reductions are deterministic: fixed-order block trees, then the block
// partials summed in block order by one block.
#pragma once
#include "common.cuh"

namespace sdr {

constexpr int kMetBS = 256;

// MetricsCollector::new (metrics.rs:124-170): a wall cell is an inside cell
// with a non-inside (or out-of-domain) face neighbour. inside == cavity mask.
__global__ void k_wall_mask(Grid g, const uint8_t* __restrict__ inside, uint8_t* __restrict__ is_wall,
                            unsigned long long* __restrict__ wall_count) {
    __shared__ uint32_t sh[33];
    size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    size_t n = (size_t)g.nx * g.ny * g.nz;
    uint32_t wall = 0;
    if (c < n) {
        if (inside[c]) {
            int i = c % g.nx, j = (c / g.nx) % g.ny, k = c / ((size_t)g.nx * g.ny);
            auto solid = [&](int a, int b, int d) {
                if (a < 0 || b < 0 || d < 0 || a >= g.nx || b >= g.ny || d >= g.nz) return true;
                return !inside[((size_t)d * g.ny + b) * g.nx + a];
            };
            wall = solid(i - 1, j, k) || solid(i + 1, j, k) || solid(i, j - 1, k) || solid(i, j + 1, k) ||
                   solid(i, j, k - 1) || solid(i, j, k + 1);
        }
        is_wall[c] = (uint8_t)wall;
    }
    uint32_t s = block_sum_u32<kMetBS>(wall, sh);
    if (threadIdx.x == 0 && s) atomicAdd(wall_count, (unsigned long long)s);
}

// Particle pass (metrics.rs:196-204 + solver.rs:884-890 + particles.rs:52-56):
// mark washed/wet wall cells; per-block max speed and sum |v|^2 in f64.
__global__ void __launch_bounds__(kMetBS) k_metrics_particles(Grid g, const float4* __restrict__ pos,
                                                              const float4* __restrict__ vel, uint32_t n,
                                                              const uint8_t* __restrict__ is_wall,
                                                              uint8_t* __restrict__ washed,
                                                              uint8_t* __restrict__ wet,
                                                              double* __restrict__ part) {
    __shared__ double sh[33];
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    double sp = 0.0, e = 0.0;
    if (p < n) {
        float4 q = pos[p];
        int c = cell_of(g, q.x, q.y, q.z);
        if (c >= 0 && is_wall[c]) {
            washed[c] = 1;
            wet[c] = 1;
        }
        float4 v = vel[p];
        double l2 = dadd(dadd(dmul((double)v.x, (double)v.x), dmul((double)v.y, (double)v.y)),
                         dmul((double)v.z, (double)v.z));
        e = l2;
        sp = __dsqrt_rn(l2);
    }
    double m = block_max<kMetBS>(sp, sh);
    double s = block_sum<kMetBS>(e, sh);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = m;
        part[2 * blockIdx.x + 1] = s;
    }
}

struct CellPart {
    double fl_max, fl_sum, ww_sum, ww_peak;
    uint32_t fl_n, ww_n, ww_art, washed;
};

// Cell pass: fluid pressure max/mean (solver.rs:859-881), washed count, and
// membrane_stats over wet wall cells (metrics.rs:238-239, 460-478); clears
// the per-frame wet mask.
__global__ void __launch_bounds__(kMetBS) k_metrics_cells(size_t n, const uint8_t* __restrict__ cells,
                                                          const double* __restrict__ p,
                                                          const uint8_t* __restrict__ washed,
                                                          uint8_t* __restrict__ wet, double cap,
                                                          CellPart* __restrict__ part) {
    __shared__ double sh[33];
    __shared__ uint32_t shu[33];
    size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    double fmaxv = 0.0, fsum = 0.0, wsum = 0.0, wpeak = 0.0;
    uint32_t fn = 0, wn = 0, wa = 0, wc = 0;
    if (c < n) {
        double pv = p[c];
        if (cells[c] == FLUID) {
            fmaxv = fmax(0.0, pv);
            fsum = pv;
            fn = 1;
        }
        if (wet[c]) {
            if (pv > cap) {
                wa = 1;
            } else {
                wsum = pv;
                wpeak = fmax(0.0, pv);
                wn = 1;
            }
            wet[c] = 0;
        }
        wc = washed[c];
    }
    CellPart r;
    r.fl_max = block_max<kMetBS>(fmaxv, sh);
    r.fl_sum = block_sum<kMetBS>(fsum, sh);
    r.ww_sum = block_sum<kMetBS>(wsum, sh);
    r.ww_peak = block_max<kMetBS>(wpeak, sh);
    r.fl_n = block_sum_u32<kMetBS>(fn, shu);
    r.ww_n = block_sum_u32<kMetBS>(wn, shu);
    r.ww_art = block_sum_u32<kMetBS>(wa, shu);
    r.washed = block_sum_u32<kMetBS>(wc, shu);
    if (threadIdx.x == 0) part[blockIdx.x] = r;
}

struct MetricsOut {
    double fl_max, fl_sum, ww_sum, ww_peak, max_speed, ke_sum;
    unsigned long long fl_n, ww_n, ww_art, washed;
};

// Block partials summed in block order by one thread (deterministic).
__global__ void k_metrics_final(const CellPart* __restrict__ cp, int ncb, const double* __restrict__ pp,
                                int npb, MetricsOut* __restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    MetricsOut o{};
    for (int b = 0; b < ncb; ++b) {
        o.fl_max = fmax(o.fl_max, cp[b].fl_max);
        o.fl_sum = dadd(o.fl_sum, cp[b].fl_sum);
        o.ww_sum = dadd(o.ww_sum, cp[b].ww_sum);
        o.ww_peak = fmax(o.ww_peak, cp[b].ww_peak);
        o.fl_n += cp[b].fl_n;
        o.ww_n += cp[b].ww_n;
        o.ww_art += cp[b].ww_art;
        o.washed += cp[b].washed;
    }
    for (int b = 0; b < npb; ++b) {
        o.max_speed = fmax(o.max_speed, pp[2 * b]);
        o.ke_sum = dadd(o.ke_sum, pp[2 * b + 1]);
    }
    *out = o;
}

// max_particles_per_cell (solver.rs:770-782) from a histogram.
__global__ void k_hist_max(const uint32_t* __restrict__ h, size_t n, unsigned int* __restrict__ out) {
    unsigned int m = 0;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        m = max(m, h[q]);
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

__global__ void k_count_fluid(const uint8_t* __restrict__ cells, size_t n,
                              unsigned long long* __restrict__ out) {
    __shared__ uint32_t sh[33];
    size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t v = (c < n && cells[c] == FLUID) ? 1u : 0u;
    uint32_t s = block_sum_u32<kMetBS>(v, sh);
    if (threadIdx.x == 0 && s) atomicAdd(out, (unsigned long long)s);
}

}  // namespace sdr
