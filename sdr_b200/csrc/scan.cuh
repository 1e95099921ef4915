// Exclusive prefix sums over u32 arrays (tile = 4096 items per 1024-thread block).
// Used for the counting-sort cell starts, order-preserving particle compaction
// (ParticleSet::retain, src/particles.rs:38-49) and the fluid-cell lists.
#pragma once
#include "common.cuh"

namespace sdr {

constexpr int kScanBS = 1024;
constexpr int kScanIPT = 4;
constexpr int kScanTile = kScanBS * kScanIPT;

// Block-wide exclusive scan of one value per thread; returns the block total.
__device__ __forceinline__ uint32_t block_exscan_u32(uint32_t v, uint32_t& excl, uint32_t* sh) {
    int l = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (l >= o) x += y;
    }
    if (l == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t s = (l < (int)(blockDim.x >> 5)) ? sh[l] : 0u;
        uint32_t t = s;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
            if (l >= o) t += y;
        }
        sh[l] = t - s;            // exclusive warp offsets
        if (l == 31) sh[32] = t;  // block total
    }
    __syncthreads();
    excl = sh[w] + x - v;
    uint32_t total = sh[32];
    __syncthreads();
    return total;
}

__device__ __forceinline__ void k_scan_tiles_body(VB vb_, const uint32_t* __restrict__ in, uint32_t n,
                                                       uint32_t* __restrict__ tile_sums) {
    __shared__ uint32_t sh[33];
    size_t base = (size_t)vb_.bid * kScanTile + (size_t)threadIdx.x * kScanIPT;
    uint32_t s = 0;
#pragma unroll
    for (int q = 0; q < kScanIPT; ++q)
        if (base + q < n) s += in[base + q];
    uint32_t ex;
    uint32_t tot = block_exscan_u32(s, ex, sh);
    if (threadIdx.x == 0) tile_sums[vb_.bid] = tot;
}
__global__ void __launch_bounds__(kScanBS) k_scan_tiles(const uint32_t* __restrict__ in, uint32_t n,
                                                       uint32_t* __restrict__ tile_sums) { k_scan_tiles_body(VB{blockIdx.x, gridDim.x}, in, n, tile_sums); }

// One block scans all tile sums (exclusive) in order; writes the grand total.
__device__ __forceinline__ void k_scan_sums_body(VB vb_, uint32_t* __restrict__ sums, uint32_t nt,
                                                      uint32_t* __restrict__ total) {
    __shared__ uint32_t sh[33];
    uint32_t carry = 0;
    for (uint32_t b = 0; b < nt; b += kScanBS) {
        uint32_t i = b + threadIdx.x;
        uint32_t v = i < nt ? sums[i] : 0u;
        uint32_t ex;
        uint32_t tot = block_exscan_u32(v, ex, sh);
        if (i < nt) sums[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0 && total) *total = carry;
}
__global__ void __launch_bounds__(kScanBS) k_scan_sums(uint32_t* __restrict__ sums, uint32_t nt,
                                                      uint32_t* __restrict__ total) { k_scan_sums_body(VB{blockIdx.x, gridDim.x}, sums, nt, total); }

__device__ __forceinline__ void k_scan_apply_body(VB vb_, const uint32_t* __restrict__ in, uint32_t n,
                                                       const uint32_t* __restrict__ tile_off,
                                                       uint32_t* __restrict__ out) {
    __shared__ uint32_t sh[33];
    size_t base = (size_t)vb_.bid * kScanTile + (size_t)threadIdx.x * kScanIPT;
    uint32_t v[kScanIPT];
    uint32_t s = 0;
#pragma unroll
    for (int q = 0; q < kScanIPT; ++q) {
        v[q] = (base + q < n) ? in[base + q] : 0u;
        s += v[q];
    }
    uint32_t ex;
    block_exscan_u32(s, ex, sh);
    uint32_t run = tile_off[vb_.bid] + ex;
#pragma unroll
    for (int q = 0; q < kScanIPT; ++q) {
        if (base + q < n) out[base + q] = run;
        run += v[q];
    }
}
__global__ void __launch_bounds__(kScanBS) k_scan_apply(const uint32_t* __restrict__ in, uint32_t n,
                                                       const uint32_t* __restrict__ tile_off,
                                                       uint32_t* __restrict__ out) { k_scan_apply_body(VB{blockIdx.x, gridDim.x}, in, n, tile_off, out); }

}  // namespace sdr
