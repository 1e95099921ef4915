// Particle-side kernels of Solver::substep (src/solver.rs:284-310):
// classify + cell keys, the P2G counting sort and fixed-order face gather,
// G2P (FLIP/PIC) fused with RK2 advection and the bounds flags, the stable
// compaction of ParticleSet::retain, and the redistribution sweeps.
#pragma once
#include "common.cuh"
#include "scan.cuh"

namespace sdr {

constexpr int kBS = 256;

// ------------------------------------------------------------------ classify
// Solver::classify (solver.rs:342-371) first half: static labels per cell.
__device__ __forceinline__ void k_base_labels_body(VB vb_, const uint8_t* __restrict__ base, uint8_t* __restrict__ cells,
                              size_t n) {
    size_t c = (size_t)vb_.bid * blockDim.x + threadIdx.x;
    if (c < n) cells[c] = base[c];
}
__global__ void k_base_labels(const uint8_t* __restrict__ base, uint8_t* __restrict__ cells,
                              size_t n) { k_base_labels_body(VB{blockIdx.x, gridDim.x}, base, cells, n); }

// Per particle: the f64 cell key of Solver::cell_of (labels, histograms) and
// the clamped cell the P2G gather bins by (from the same f64 grid coordinate
// the gather's weights use, so every contribution lands in the gathered stencil).
// With mark_fluid, also the second half of classify: Air cells holding a
// particle that is not in the outlet become Fluid (solver.rs:362-370).
__device__ __forceinline__ void k_classify_keys_body(VB vb_, Grid g, const float4* __restrict__ pos, uint32_t n,
                                int has_outlet, Aabb outlet, int mark_fluid,
                                uint8_t* __restrict__ cells, int* __restrict__ key_cell,
                                uint32_t* __restrict__ key_sort, uint32_t* __restrict__ hist_valid,
                                uint32_t* __restrict__ hist_sort) {
    uint32_t p = vb_.bid * blockDim.x + threadIdx.x;
    if (p >= n) return;
    float4 q = pos[p];
    int c = cell_of(g, q.x, q.y, q.z);
    key_cell[p] = c;
    if (c >= 0) {
        atomicAdd(&hist_valid[c], 1u);
        if (mark_fluid && cells[c] == AIR &&
            !(has_outlet && aabb_contains(outlet, q.x, q.y, q.z)))
            cells[c] = FLUID;  // benign race: every writer stores FLUID
    }
    double lx = ddiv(dsub((double)q.x, g.ox), g.dx), ly = ddiv(dsub((double)q.y, g.oy), g.dx),
           lz = ddiv(dsub((double)q.z, g.oz), g.dx);
    int i = (lx > 0.0) ? (int)fmin(floor(lx), (double)(g.nx - 1)) : 0;
    int j = (ly > 0.0) ? (int)fmin(floor(ly), (double)(g.ny - 1)) : 0;
    int k = (lz > 0.0) ? (int)fmin(floor(lz), (double)(g.nz - 1)) : 0;
    uint32_t ks = ((uint32_t)k * g.ny + j) * g.nx + i;
    key_sort[p] = ks;
    atomicAdd(&hist_sort[ks], 1u);
}
__global__ void k_classify_keys(Grid g, const float4* __restrict__ pos, uint32_t n,
                                int has_outlet, Aabb outlet, int mark_fluid,
                                uint8_t* __restrict__ cells, int* __restrict__ key_cell,
                                uint32_t* __restrict__ key_sort, uint32_t* __restrict__ hist_valid,
                                uint32_t* __restrict__ hist_sort) { k_classify_keys_body(VB{blockIdx.x, gridDim.x}, g, pos, n, has_outlet, outlet, mark_fluid, cells, key_cell, key_sort, hist_valid, hist_sort); }

// ------------------------------------------------------------------ counting sort
// Slot assignment within each cell segment (start from the exclusive scan).
__device__ __forceinline__ void k_sort_scatter_body(VB vb_, const uint32_t* __restrict__ key, uint32_t n,
                               uint32_t* __restrict__ fill, uint32_t* __restrict__ perm) {
    uint32_t p = vb_.bid * blockDim.x + threadIdx.x;
    if (p >= n) return;
    uint32_t s = atomicAdd(&fill[key[p]], 1u);
    perm[s] = p;
}
__global__ void k_sort_scatter(const uint32_t* __restrict__ key, uint32_t n,
                               uint32_t* __restrict__ fill, uint32_t* __restrict__ perm) { k_sort_scatter_body(VB{blockIdx.x, gridDim.x}, key, n, fill, perm); }

// Make each segment ascending in particle index, so the permutation equals a
// stable counting sort (bit-exact vs a CPU stable sort of the same keys) and
// the gather's summation order is fixed. Short segments: insertion sort by
// one thread; long ones are queued for k_sort_long.
__device__ __forceinline__ void k_sort_segments_body(VB vb_, const uint32_t* __restrict__ start, uint32_t ncell,
                                uint32_t* __restrict__ perm, uint32_t* __restrict__ long_list,
                                uint32_t* __restrict__ long_count) {
    uint32_t c = vb_.bid * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    uint32_t a = start[c], b = start[c + 1];
    uint32_t len = b - a;
    if (len < 2) return;
    if (len > 48) {
        uint32_t s = atomicAdd(long_count, 1u);
        long_list[s] = c;
        return;
    }
    for (uint32_t x = a + 1; x < b; ++x) {
        uint32_t v = perm[x];
        uint32_t y = x;
        while (y > a && perm[y - 1] > v) {
            perm[y] = perm[y - 1];
            --y;
        }
        perm[y] = v;
    }
}
__global__ void k_sort_segments(const uint32_t* __restrict__ start, uint32_t ncell,
                                uint32_t* __restrict__ perm, uint32_t* __restrict__ long_list,
                                uint32_t* __restrict__ long_count) { k_sort_segments_body(VB{blockIdx.x, gridDim.x}, start, ncell, perm, long_list, long_count); }

// Rank sort of long segments (indices are distinct): one block per segment.
__device__ __forceinline__ void k_sort_long_body(VB vb_, const uint32_t* __restrict__ start, const uint32_t* __restrict__ long_list,
                            const uint32_t* __restrict__ long_count, uint32_t* __restrict__ perm,
                            uint32_t* __restrict__ tmp) {
    uint32_t nl = *long_count;
    for (uint32_t q = vb_.bid; q < nl; q += vb_.nb) {
        uint32_t c = long_list[q];
        uint32_t a = start[c], b = start[c + 1];
        for (uint32_t x = a + threadIdx.x; x < b; x += blockDim.x) {
            uint32_t v = perm[x];
            uint32_t r = 0;
            for (uint32_t y = a; y < b; ++y) r += perm[y] < v;
            tmp[a + r] = v;
        }
        __syncthreads();
        for (uint32_t x = a + threadIdx.x; x < b; x += blockDim.x) perm[x] = tmp[x];
        __syncthreads();
    }
}
__global__ void k_sort_long(const uint32_t* __restrict__ start, const uint32_t* __restrict__ long_list,
                            const uint32_t* __restrict__ long_count, uint32_t* __restrict__ perm,
                            uint32_t* __restrict__ tmp) { k_sort_long_body(VB{blockIdx.x, gridDim.x}, start, long_list, long_count, perm, tmp); }

// ------------------------------------------------------------------ P2G gather
// Sorted particle records for the gather: the f64 grid coordinate
// (p - origin)/dx of Solver's u/v/w_coords (grid.rs:161-175) and the f32 velocity.
__device__ __forceinline__ void k_sorted_records_body(VB vb_, Grid g, const float4* __restrict__ pos, const float4* __restrict__ vel,
                                 const uint32_t* __restrict__ perm, uint32_t n, double4* __restrict__ lrec,
                                 float4* __restrict__ vrec) {
    uint32_t s = vb_.bid * blockDim.x + threadIdx.x;
    if (s >= n) return;
    uint32_t p = perm[s];
    float4 q = pos[p];
    lrec[s] = make_double4(ddiv(dsub((double)q.x, g.ox), g.dx), ddiv(dsub((double)q.y, g.oy), g.dx),
                           ddiv(dsub((double)q.z, g.oz), g.dx), 0.0);
    vrec[s] = vel[p];
}
__global__ void k_sorted_records(Grid g, const float4* __restrict__ pos, const float4* __restrict__ vel,
                                 const uint32_t* __restrict__ perm, uint32_t n, double4* __restrict__ lrec,
                                 float4* __restrict__ vrec) { k_sorted_records_body(VB{blockIdx.x, gridDim.x}, g, pos, vel, perm, n, lrec, vrec); }

struct P2GArgs {
    Grid g;
    const double4* lrec;
    const float4* vrec;
    const uint32_t* start;  // ncell + 1
    float* u;
    float* v;
    float* w;
    float* su;
    float* sv;
    float* sw;
    const uint8_t* cells;  // for enforce_solid_faces (may be null)
    double gdt[3];         // gravity * dt per component (0 = skip)
    int add_forces;
    int enforce;
};

// Is face (i,j,k) of a component next to a Solid cell or the domain edge?
// (pressure.rs:243-281)
__device__ __forceinline__ bool solid_at(const Grid& g, const uint8_t* cells, int i, int j, int k) {
    if (i < 0 || j < 0 || k < 0 || i >= g.nx || j >= g.ny || k >= g.nz) return true;
    return cells[((size_t)k * g.ny + j) * g.nx + i] == SOLID;
}

// Flat node index -> (i, j, k) over (nx+1) x (ny+1) x (nz+1).
__device__ __forceinline__ bool node_of(const Grid& g, size_t t, int& i, int& j, int& k) {
    size_t nxp = (size_t)g.nx + 1, nyp = (size_t)g.ny + 1;
    if (t >= nxp * nyp * ((size_t)g.nz + 1)) return false;
    i = (int)(t % nxp);
    j = (int)((t / nxp) % nyp);
    k = (int)(t / (nxp * nyp));
    return true;
}

// clamp_base (grid.rs:25-34) in f64 and the weight of node `i` (0 if not a corner).
__device__ __forceinline__ double corner_w(double gcoord, int n, int node) {
    int i0;
    double f;
    if (!(gcoord > 0.0)) {
        i0 = 0;
        f = 0.0;
    } else if (gcoord >= (double)(n - 1)) {
        i0 = n - 2;
        f = 1.0;
    } else {
        double fl = floor(gcoord);
        i0 = (int)fl;
        f = dsub(gcoord, fl);
    }
    int d = node - i0;
    return d == 0 ? dsub(1.0, f) : (d == 1 ? f : -1.0);
}

// Normalise (solver.rs:944-952), save the FLIP copy (save_grid), optionally
// add gravity and zero solid faces: the faces owned by node (i, j, k).
__device__ __forceinline__ void p2g_store(const P2GArgs& a, int i, int j, int k, bool hu, bool hv, bool hw,
                                          double su, double wu, double sv, double wv, double sw, double ww) {
    const Grid& g = a.g;
    if (hu) {
        size_t f = ((size_t)k * g.ny + j) * (g.nx + 1) + i;
        float val = wu > 1e-12 ? (float)ddiv(su, wu) : 0.0f;
        a.su[f] = val;
        if (a.add_forces && a.gdt[0] != 0.0) val = (float)dadd((double)val, a.gdt[0]);
        if (a.enforce && (solid_at(g, a.cells, i - 1, j, k) || solid_at(g, a.cells, i, j, k))) val = 0.0f;
        a.u[f] = val;
    }
    if (hv) {
        size_t f = ((size_t)k * (g.ny + 1) + j) * g.nx + i;
        float val = wv > 1e-12 ? (float)ddiv(sv, wv) : 0.0f;
        a.sv[f] = val;
        if (a.add_forces && a.gdt[1] != 0.0) val = (float)dadd((double)val, a.gdt[1]);
        if (a.enforce && (solid_at(g, a.cells, i, j - 1, k) || solid_at(g, a.cells, i, j, k))) val = 0.0f;
        a.v[f] = val;
    }
    if (hw) {
        size_t f = ((size_t)k * g.ny + j) * g.nx + i;
        float val = ww > 1e-12 ? (float)ddiv(sw, ww) : 0.0f;
        a.sw[f] = val;
        if (a.add_forces && a.gdt[2] != 0.0) val = (float)dadd((double)val, a.gdt[2]);
        if (a.enforce && (solid_at(g, a.cells, i, j, k - 1) || solid_at(g, a.cells, i, j, k))) val = 0.0f;
        a.w[f] = val;
    }
}


// P2G, first pass: one thread per grid node (i,j,k) in [0,nx]x[0,ny]x[0,nz]
// (the node owns the u, v and w faces with that index). A node with no
// particle in the 27 cells around it gets its faces at once (all sums +0);
// the others are queued for k_p2g.
__device__ __forceinline__ void k_p2g_nodes_body(VB vb_, P2GArgs a, uint32_t* __restrict__ list,
                                                   uint32_t* __restrict__ count) {
    const Grid& g = a.g;
    const size_t t = (size_t)vb_.bid * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!node_of(g, t, i, j, k)) return;
    uint32_t cnt = 0;
    const int ci0 = max(i - 1, 0), ci1 = min(i + 1, g.nx - 1);
    for (int ck = max(k - 1, 0); ck <= min(k + 1, g.nz - 1); ++ck)
        for (int cj = max(j - 1, 0); cj <= min(j + 1, g.ny - 1); ++cj) {
            const uint32_t c = ((uint32_t)ck * g.ny + cj) * g.nx;
            cnt += a.start[c + ci1 + 1] - a.start[c + ci0];
        }
    if (cnt) list[atomicAdd(count, 1u)] = (uint32_t)t;
    else p2g_store(a, i, j, k, j < g.ny && k < g.nz, i < g.nx && k < g.nz, i < g.nx && j < g.ny, 0, 0, 0, 0, 0, 0);
}
__global__ void __launch_bounds__(kBS) k_p2g_nodes(P2GArgs a, uint32_t* __restrict__ list,
                                                   uint32_t* __restrict__ count) { k_p2g_nodes_body(VB{blockIdx.x, gridDim.x}, a, list, count); }

// P2G gather of the queued nodes, eight lanes each. The lanes split the
// particles of the 27 cells around the node — for each (k, j) the three cells
// i-1..i+1 are one contiguous run of the sorted records, and lane l takes
// every eighth record of each run from the l-th — accumulating the
// trilinear_scatter weights (grid.rs:52-88, w = wx*wy*wz) in f64; a fixed
// xor tree of shuffles then adds the eight partial sums (the same bits in
// every lane: each step adds the same pair). The order is fixed, so the
// result is deterministic; busy nodes (the jet clump) do not hold their warp
// for hundreds of sequential particles. The loop over the queue takes the
// same trips in every thread, so the shuffles always see whole warps.
constexpr int kP2GLanes = 8;
__device__ __forceinline__ void k_p2g_body(VB vb_, P2GArgs a, const uint32_t* __restrict__ list,
                                             const uint32_t* __restrict__ count) {
    const Grid& g = a.g;
    const uint32_t nq = *count;
    const uint32_t groups = (uint32_t)(vb_.nb * blockDim.x / kP2GLanes);
    const uint32_t gid = (uint32_t)((vb_.bid * blockDim.x + threadIdx.x) / kP2GLanes);
    const int lane = (int)(threadIdx.x % kP2GLanes);
    for (uint32_t base = 0; base < nq; base += groups) {
        const uint32_t h = base + gid;
        int i = 0, j = 0, k = 0;
        const bool node = h < nq && node_of(g, list[min(h, nq - 1)], i, j, k);
        const bool hu = node && j < g.ny && k < g.nz, hv = node && i < g.nx && k < g.nz,
                   hw = node && i < g.nx && j < g.ny;
        double su = 0, wu = 0, sv = 0, wv = 0, sw = 0, ww = 0;
        const int ci0 = max(i - 1, 0), ci1 = min(i + 1, g.nx - 1);
        for (int ck = max(k - 1, 0); node && ck <= min(k + 1, g.nz - 1); ++ck)
            for (int cj = max(j - 1, 0); cj <= min(j + 1, g.ny - 1); ++cj) {
                uint32_t c = ((uint32_t)ck * g.ny + cj) * g.nx;
                uint32_t s0 = a.start[c + ci0], s1 = a.start[c + ci1 + 1];
                for (uint32_t s = s0 + lane; s < s1; s += kP2GLanes) {
                    double4 l = a.lrec[s];
                    float4 vel = a.vrec[s];
                    if (hu) {
                        double wx = corner_w(l.x, g.nx + 1, i), wy = corner_w(l.y - 0.5, g.ny, j),
                               wz = corner_w(l.z - 0.5, g.nz, k);
                        if (wx >= 0.0 && wy >= 0.0 && wz >= 0.0) {
                            double wgt = dmul(dmul(wx, wy), wz);
                            su = dadd(su, dmul(wgt, (double)vel.x));
                            wu = dadd(wu, wgt);
                        }
                    }
                    if (hv) {
                        double wx = corner_w(l.x - 0.5, g.nx, i), wy = corner_w(l.y, g.ny + 1, j),
                               wz = corner_w(l.z - 0.5, g.nz, k);
                        if (wx >= 0.0 && wy >= 0.0 && wz >= 0.0) {
                            double wgt = dmul(dmul(wx, wy), wz);
                            sv = dadd(sv, dmul(wgt, (double)vel.y));
                            wv = dadd(wv, wgt);
                        }
                    }
                    if (hw) {
                        double wx = corner_w(l.x - 0.5, g.nx, i), wy = corner_w(l.y - 0.5, g.ny, j),
                               wz = corner_w(l.z, g.nz + 1, k);
                        if (wx >= 0.0 && wy >= 0.0 && wz >= 0.0) {
                            double wgt = dmul(dmul(wx, wy), wz);
                            sw = dadd(sw, dmul(wgt, (double)vel.z));
                            ww = dadd(ww, wgt);
                        }
                    }
                }
            }
#pragma unroll
        for (int o = kP2GLanes / 2; o > 0; o >>= 1) {
            su = dadd(su, __shfl_xor_sync(0xffffffffu, su, o, kP2GLanes));
            wu = dadd(wu, __shfl_xor_sync(0xffffffffu, wu, o, kP2GLanes));
            sv = dadd(sv, __shfl_xor_sync(0xffffffffu, sv, o, kP2GLanes));
            wv = dadd(wv, __shfl_xor_sync(0xffffffffu, wv, o, kP2GLanes));
            sw = dadd(sw, __shfl_xor_sync(0xffffffffu, sw, o, kP2GLanes));
            ww = dadd(ww, __shfl_xor_sync(0xffffffffu, ww, o, kP2GLanes));
        }
        if (node && lane == 0) p2g_store(a, i, j, k, hu, hv, hw, su, wu, sv, wv, sw, ww);
    }
}
__global__ void __launch_bounds__(kBS) k_p2g(P2GArgs a, const uint32_t* __restrict__ list,
                                             const uint32_t* __restrict__ count) { k_p2g_body(VB{blockIdx.x, gridDim.x}, a, list, count); }

// Solver::add_forces (solver.rs:593-604) on its own (phase mode).
__device__ __forceinline__ void k_add_forces_body(VB vb_, float* __restrict__ f, size_t n, double gdt) {
    size_t q = (size_t)vb_.bid * blockDim.x + threadIdx.x;
    if (q < n) f[q] = (float)dadd((double)f[q], gdt);
}
__global__ void k_add_forces(float* __restrict__ f, size_t n, double gdt) { k_add_forces_body(VB{blockIdx.x, gridDim.x}, f, n, gdt); }

// enforce_solid_faces (pressure.rs:243-281) on its own (phase mode): one
// thread per node, owning the u/v/w faces with that index.
__device__ __forceinline__ void k_enforce_solid_body(VB vb_, Grid g, const uint8_t* __restrict__ cells, float* __restrict__ u,
                                float* __restrict__ v, float* __restrict__ w) {
    int i, j, k;
    if (!node_of(g, (size_t)vb_.bid * blockDim.x + threadIdx.x, i, j, k)) return;
    if (j < g.ny && k < g.nz && (solid_at(g, cells, i - 1, j, k) || solid_at(g, cells, i, j, k)))
        u[((size_t)k * g.ny + j) * (g.nx + 1) + i] = 0.0f;
    if (i < g.nx && k < g.nz && (solid_at(g, cells, i, j - 1, k) || solid_at(g, cells, i, j, k)))
        v[((size_t)k * (g.ny + 1) + j) * g.nx + i] = 0.0f;
    if (i < g.nx && j < g.ny && (solid_at(g, cells, i, j, k - 1) || solid_at(g, cells, i, j, k)))
        w[((size_t)k * g.ny + j) * g.nx + i] = 0.0f;
}
__global__ void k_enforce_solid(Grid g, const uint8_t* __restrict__ cells, float* __restrict__ u,
                                float* __restrict__ v, float* __restrict__ w) { k_enforce_solid_body(VB{blockIdx.x, gridDim.x}, g, cells, u, v, w); }

// ------------------------------------------------------------------ G2P + advect
struct MoveArgs {
    Grid g;
    Sdf sdf;
    float4* pos;
    float4* vel;
    const uint32_t* order;  // processing order (sorted slots -> particle), or null
    uint32_t n;
    Faces f;         // projected, extrapolated faces
    Faces saved;     // post-P2G faces
    float flip;      // clamp(flip_ratio, 0, 1)
    float dt;
    int do_g2p;
    int do_advect;
    int do_bounds;   // write keep/drained flags
    Aabb bb;         // solid.bounds()
    int has_outlet;
    Aabb outlet;
    float cull_phi;  // 0.5 * solid.dx
    uint32_t* keep;  // 1 = keep (ParticleSet::retain predicate)
    uint32_t* drained;
};

// Bounds predicate of enforce_particle_bounds (solver.rs:736-755).
__device__ __forceinline__ void bounds_flags(const MoveArgs& a, float3 p, uint32_t& keep,
                                             uint32_t& drained) {
    drained = 0;
    if (!aabb_contains(a.bb, p.x, p.y, p.z)) {
        keep = 0;
        return;
    }
    if (a.has_outlet && aabb_contains(a.outlet, p.x, p.y, p.z)) {
        keep = 0;
        drained = 1;
        return;
    }
    keep = sdf_sample(a.sdf, p.x, p.y, p.z) < a.cull_phi ? 1u : 0u;
}

// Solver::g2p (solver.rs:650-677) fused with Solver::advect (solver.rs:693-711)
// and the bounds predicate. Both read the pre-advection position and the same
// grid, so velocity_at(p0) is shared. Particles are visited in sorted-cell
// order so neighbouring threads read neighbouring faces.
__device__ __forceinline__ void k_g2p_advect_body(VB vb_, MoveArgs a) {
    uint32_t t = vb_.bid * blockDim.x + threadIdx.x;
    if (t >= a.n) return;
    uint32_t p = a.order ? a.order[t] : t;
    const Grid& g = a.g;
    float4 q = a.pos[p];
    float3 p0 = make_float3(q.x, q.y, q.z);
    float3 v0 = velocity_at(g, a.f, p0.x, p0.y, p0.z);
    if (a.do_g2p) {
        float lx = (p0.x - g.oxf) / g.dxf, ly = (p0.y - g.oyf) / g.dxf, lz = (p0.z - g.ozf) / g.dxf;
        float dvx = trilerp_diff(a.f.u, a.saved.u, g.nx + 1, g.ny, g.nz, lx, ly - 0.5f, lz - 0.5f);
        float dvy = trilerp_diff(a.f.v, a.saved.v, g.nx, g.ny + 1, g.nz, lx - 0.5f, ly, lz - 0.5f);
        float dvz = trilerp_diff(a.f.w, a.saved.w, g.nx, g.ny, g.nz + 1, lx - 0.5f, ly - 0.5f, lz);
        float4 v = a.vel[p];
        float pic = 1.0f - a.flip;
        v.x = (v.x + dvx) * a.flip + v0.x * pic;
        v.y = (v.y + dvy) * a.flip + v0.y * pic;
        v.z = (v.z + dvz) * a.flip + v0.z * pic;
        a.vel[p] = v;
    }
    float3 pn = p0;
    if (a.do_advect) {
        float h = 0.5f * a.dt;
        float3 mid = make_float3(p0.x + v0.x * h, p0.y + v0.y * h, p0.z + v0.z * h);
        float3 vm = velocity_at(g, a.f, mid.x, mid.y, mid.z);
        float3 st = make_float3(vm.x * a.dt, vm.y * a.dt, vm.z * a.dt);
        float len = sqrtf(st.x * st.x + st.y * st.y + st.z * st.z);
        if (len > g.dxf) {
            float sc = g.dxf / len;
            st = make_float3(st.x * sc, st.y * sc, st.z * sc);
        }
        float3 c = project_inside(a.sdf, 0.5f * g.dxf, make_float3(p0.x + st.x, p0.y + st.y, p0.z + st.z));
        if (sdf_sample(a.sdf, c.x, c.y, c.z) <= 0.0f) pn = c;
        a.pos[p] = make_float4(pn.x, pn.y, pn.z, 0.0f);
    }
    if (a.do_bounds) {
        uint32_t k, d;
        bounds_flags(a, pn, k, d);
        a.keep[p] = k;
        a.drained[p] = d;
    }
}
__global__ void __launch_bounds__(kBS) k_g2p_advect(MoveArgs a) { k_g2p_advect_body(VB{blockIdx.x, gridDim.x}, a); }

// Bounds flags alone (phase mode, after an external position change).
__device__ __forceinline__ void k_bounds_flags_body(VB vb_, MoveArgs a) {
    uint32_t p = vb_.bid * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    float4 q = a.pos[p];
    uint32_t k, d;
    bounds_flags(a, make_float3(q.x, q.y, q.z), k, d);
    a.keep[p] = k;
    a.drained[p] = d;
}
__global__ void k_bounds_flags(MoveArgs a) { k_bounds_flags_body(VB{blockIdx.x, gridDim.x}, a); }

// Stable scatter of kept particles (ParticleSet::retain, particles.rs:38-49)
// plus the drained/culled tallies.
__device__ __forceinline__ void k_compact_body(VB vb_, const float4* __restrict__ pos, const float4* __restrict__ vel,
                          const uint32_t* __restrict__ keep, const uint32_t* __restrict__ drained,
                          const uint32_t* __restrict__ off, uint32_t n, float4* __restrict__ pos2,
                          float4* __restrict__ vel2, unsigned long long* __restrict__ counters) {
    __shared__ uint32_t sh[33];
    uint32_t p = vb_.bid * blockDim.x + threadIdx.x;
    uint32_t d = 0, c = 0;
    if (p < n) {
        if (keep[p]) {
            uint32_t o = off[p];
            pos2[o] = pos[p];
            vel2[o] = vel[p];
        } else {
            d = drained[p];
            c = 1 - d;
        }
    }
    uint32_t sd = block_sum_u32<kBS>(d, sh);
    uint32_t sc = block_sum_u32<kBS>(c, sh);
    if (threadIdx.x == 0) {
        if (sd) atomicAdd(&counters[0], (unsigned long long)sd);
        if (sc) atomicAdd(&counters[1], (unsigned long long)sc);
    }
}
__global__ void k_compact(const float4* __restrict__ pos, const float4* __restrict__ vel,
                          const uint32_t* __restrict__ keep, const uint32_t* __restrict__ drained,
                          const uint32_t* __restrict__ off, uint32_t n, float4* __restrict__ pos2,
                          float4* __restrict__ vel2, unsigned long long* __restrict__ counters) { k_compact_body(VB{blockIdx.x, gridDim.x}, pos, vel, keep, drained, off, n, pos2, vel2, counters); }

// ------------------------------------------------------------------ redistribute
// Solver::redistribute (solver.rs:454-557). Facts the GPU form relies on:
//  * a cell sheds only while its count exceeds the cap, and only cells over
//    the cap at the start of a sweep can ever exceed it (receivers stop at the
//    cap), so only particles in those cells can move;
//  * decisions read counts only; positions/velocities of moved particles are
//    functions of (index, destination cell) and can be written afterwards;
//  * a sweep that moves nothing leaves the state unchanged, so every later
//    sweep of the substep moves nothing either.
// Per sweep: histogram -> append candidates -> one block sorts them by index,
// replays the sequential decisions in shared memory, and applies the moves.

struct RedistState {
    uint32_t ncand;   // candidates appended this sweep
    uint32_t active;  // 0 once a sweep made no move (later sweeps are no-ops)
    uint32_t nmoves;  // moves of the last sweep
    uint32_t err;
    unsigned long long moves_total;
    unsigned long long cand_total;   // candidates replayed, all sweeps so far
    unsigned long long sweeps_total;  // replay sweeps that ran
    unsigned long long long_total;    // of those, sweeps past the shared-memory list
    uint32_t par;         // 1: the list is long; k_redist_par decides and applies this sweep
    uint32_t round_base;  // claim stamps used so far by k_redist_par (grows across sweeps)
    uint32_t nmoves_par;  // moves appended by k_redist_par this sweep
    uint32_t pad;
    unsigned long long rounds_total;  // decision rounds of long lists, all sweeps so far
    uint32_t pend_n[2];               // entries of the two pending lists of k_redist_par's rounds
};

__device__ __forceinline__ void k_redist_hist_n_body(VB vb_, Grid g, const float4* __restrict__ pos, const uint32_t* __restrict__ n_dev,
                                const RedistState* __restrict__ rs, int* __restrict__ key_cell,
                                uint32_t* __restrict__ count) {
    if (!rs->active) return;
    uint32_t p = vb_.bid * blockDim.x + threadIdx.x;
    if (p >= *n_dev) return;
    float4 q = pos[p];
    int c = cell_of(g, q.x, q.y, q.z);
    key_cell[p] = c;
    if (c >= 0) atomicAdd(&count[c], 1u);
}
__global__ void k_redist_hist_n(Grid g, const float4* __restrict__ pos, const uint32_t* __restrict__ n_dev,
                                const RedistState* __restrict__ rs, int* __restrict__ key_cell,
                                uint32_t* __restrict__ count) { k_redist_hist_n_body(VB{blockIdx.x, gridDim.x}, g, pos, n_dev, rs, key_cell, count); }

// Particles in over-cap cells, appended in arbitrary order (sorted later).
// A particle is left out when no face neighbour of its cell is an in-cavity
// cell below the cap at the start of the sweep: within a sweep a cell only
// receives while below the cap and a source never drains below it, so such a
// cell never gains a receiver and the reference loop (solver.rs:476-555)
// leaves every one of its particles where it is. The moves are unchanged.
__device__ __forceinline__ void k_redist_append_body(VB vb_, Grid g, const int* __restrict__ key_cell, const uint32_t* __restrict__ count,
                                const uint8_t* __restrict__ cavity, const uint32_t* __restrict__ n_dev,
                                uint32_t cap, RedistState* __restrict__ rs, uint32_t* __restrict__ cand,
                                uint32_t cand_cap) {
    if (!rs->active) return;
    uint32_t p = vb_.bid * blockDim.x + threadIdx.x;
    if (p >= *n_dev) return;
    int c = key_cell[p];
    if (c < 0 || count[c] <= cap) return;
    const int i = c % g.nx, j = (c / g.nx) % g.ny, k = c / (g.nx * g.ny);
    const int sxy = g.nx * g.ny;
    const int nb[6] = {i > 0 ? c - 1 : -1, i + 1 < g.nx ? c + 1 : -1, j > 0 ? c - g.nx : -1,
                       j + 1 < g.ny ? c + g.nx : -1, k > 0 ? c - sxy : -1, k + 1 < g.nz ? c + sxy : -1};
    bool room = false;
#pragma unroll
    for (int q = 0; q < 6; ++q) room |= nb[q] >= 0 && cavity[nb[q]] && count[nb[q]] < cap;
    if (!room) return;
    uint32_t s = atomicAdd(&rs->ncand, 1u);
    if (s < cand_cap) cand[s] = p;
}
__global__ void k_redist_append(Grid g, const int* __restrict__ key_cell, const uint32_t* __restrict__ count,
                                const uint8_t* __restrict__ cavity, const uint32_t* __restrict__ n_dev,
                                uint32_t cap, RedistState* __restrict__ rs, uint32_t* __restrict__ cand,
                                uint32_t cand_cap) { k_redist_append_body(VB{blockIdx.x, gridDim.x}, g, key_cell, count, cavity, n_dev, cap, rs, cand, cand_cap); }

constexpr int kRedistTable = 4096;   // shared-memory hash slots (power of two)
constexpr int kRedistProbes = 64;    // linear probes before a cell counts as not fitting the table
constexpr int kRedistBS = 1024;
constexpr int kRedistSmemCand = 8192;  // candidates sorted and replayed in shared memory
constexpr uint32_t kResolved = 0x80000000u;  // candidate-list flag: decided (particle indices are < 2^31)
// A shared-memory round costs about as much as one thread deciding this many
// candidates in index order: rounds that decide fewer hand the rest to thread 0.
constexpr uint32_t kRoundsMinDecided = 32;

struct RedistArgs {
    Grid g;
    Sdf sdf;
    Faces f;
    float4* pos;
    float4* vel;
    const int* key_cell;
    uint32_t* count;         // histogram at sweep start (k_redist_par's rounds update it)
    const uint8_t* cavity;
    uint32_t* cand;          // candidate particles in append order (each decider sorts them in place)
    uint32_t cand_cap;
    uint32_t n_upper;        // bound on the particle count (and on every candidate index)
    uint32_t cap;
    double down[6];          // dir . gdir for -x,+x,-y,+y,-z,+z (f64, solver.rs:490-511)
    uint32_t* moves;         // pairs (particle, destination cell)
    RedistState* rs;
    unsigned long long* claim;  // per cell: the latest claim stamp (k_redist_par); zero at allocation
    int rounds;                 // short lists: parallel rounds (1) or one thread in index order (0)
    double* slots;              // unused by the rounds (kept for the launch layout)
    uint32_t* pend;             // 2 x cand_cap: the rounds' pending unit heads, double-buffered
    uint32_t* bits;             // (n_upper + 31) / 32 words: the long list's particle-index bitmap
};

// A move: the particle goes near the destination centre with its index-keyed
// jitter (hash_jitter, solver.rs:916-930), pushed inside, with the local grid
// velocity (solver.rs:545-554).
__device__ __forceinline__ void redist_apply_move(const RedistArgs& a, uint32_t p, uint32_t c) {
    const Grid& g = a.g;
    int i = c % g.nx, j = (c / g.nx) % g.ny, k = c / (g.nx * g.ny);
    uint64_t key = p;
    double jx = jitter_mix(key * 3), jy = jitter_mix(key * 3 + 1), jz = jitter_mix(key * 3 + 2);
    double cx = dadd(g.ox, dmul((double)i + 0.5, g.dx));
    double cy = dadd(g.oy, dmul((double)j + 0.5, g.dx));
    double cz = dadd(g.oz, dmul((double)k + 0.5, g.dx));
    float3 q = make_float3((float)dadd(cx, dmul(jx, g.dx)), (float)dadd(cy, dmul(jy, g.dx)),
                           (float)dadd(cz, dmul(jz, g.dx)));
    q = project_inside(a.sdf, 0.5f * g.dxf, q);
    float3 v = velocity_at(g, a.f, q.x, q.y, q.z);
    a.pos[p] = make_float4(q.x, q.y, q.z, 0.0f);
    a.vel[p] = make_float4(v.x, v.y, v.z, 0.0f);
}

__device__ __forceinline__ uint32_t rd_hash(uint32_t c) { return (c * 2654435761u) & (kRedistTable - 1); }

// One block per sweep: sort the candidates by particle index, insert every
// referenced cell into a shared hash table, replay the reference's sequential
// loop (solver.rs:476-555) in rounds and on thread 0, then apply the moves
// (solver.rs:545-554) with all threads. A list too long for shared memory, or
// whose cells do not fit the table, goes to k_redist_par (the next launch).
__device__ __forceinline__ void k_redist_replay_body(VB vb_, RedistArgs a) {
    extern __shared__ __align__(16) unsigned char rsm[];
    unsigned long long* tclaim = (unsigned long long*)rsm;  // kRedistTable: claim stamps of the rounds
    int* tkey = (int*)(tclaim + kRedistTable);              // kRedistTable
    uint32_t* tcnt = (uint32_t*)(tkey + kRedistTable);      // kRedistTable
    uint32_t* scand = tcnt + kRedistTable;                  // kRedistSmemCand
    short* slots = (short*)(scand + kRedistSmemCand);       // 7 per candidate
    uint8_t* tcav = (uint8_t*)(slots + 7 * kRedistSmemCand);  // kRedistTable
    __shared__ int overflow;
    __shared__ uint32_t s_nm;
    __shared__ uint32_t s_dec[2];  // candidates decided in the current and the next round
    RedistState* rs = a.rs;
    if (!rs->active) return;
    const uint32_t nc_all = rs->ncand;
    if (nc_all > a.cand_cap) {
        if (threadIdx.x == 0) atomicOr(&rs->err, 1u);
        return;
    }
    const uint32_t nc = nc_all;
    const Grid& g = a.g;
    const bool in_smem = nc <= (uint32_t)kRedistSmemCand;
    // ---- sort candidates ascending (indices are distinct)
    if (in_smem) {
        uint32_t np2 = 1;
        while (np2 < nc) np2 <<= 1;
        for (uint32_t t = threadIdx.x; t < np2; t += blockDim.x) scand[t] = t < nc ? a.cand[t] : 0xffffffffu;
        __syncthreads();
        for (uint32_t k = 2; k <= np2; k <<= 1)
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t t = threadIdx.x; t < np2; t += blockDim.x) {
                    uint32_t o = t ^ j;
                    if (o > t) {
                        uint32_t x = scand[t], y = scand[o];
                        bool up = (t & k) == 0;
                        if ((x > y) == up) {
                            scand[t] = y;
                            scand[o] = x;
                        }
                    }
                }
                __syncthreads();
            }
    } else {
        // Long lists go to k_redist_par (the next launch) in append order: it
        // puts them in index order over all its CTAs.
        if (threadIdx.x == 0) rs->par = 1;
        return;
    }
    const uint32_t* cl = in_smem ? scand : a.cand;
    // ---- hash table of referenced cells
    for (int s = threadIdx.x; s < kRedistTable; s += blockDim.x) {
        tkey[s] = -1;
        tclaim[s] = 0ull;
    }
    if (threadIdx.x == 0) {
        overflow = in_smem ? 0 : 1;
        s_nm = 0;
        s_dec[0] = s_dec[1] = 0;
    }
    __syncthreads();
    if (in_smem) {
        for (uint32_t m = threadIdx.x; m < nc; m += blockDim.x) {
            if (*(volatile int*)&overflow) break;  // the list goes to k_redist_par
            int c = a.key_cell[cl[m]];
            int i = c % g.nx, j = (c / g.nx) % g.ny, k = c / (g.nx * g.ny);
            int nb[7] = {c, i > 0 ? c - 1 : -1, i + 1 < g.nx ? c + 1 : -1, j > 0 ? c - g.nx : -1,
                         j + 1 < g.ny ? c + g.nx : -1, k > 0 ? c - g.nx * g.ny : -1,
                         k + 1 < g.nz ? c + g.nx * g.ny : -1};
            for (int q = 0; q < 7; ++q) {
                int slot = -1;
                if (nb[q] >= 0) {
                    uint32_t h = rd_hash((uint32_t)nb[q]);
                    for (int probe = 0; probe < kRedistProbes; ++probe) {
                        int prev = atomicCAS(&tkey[h], -1, nb[q]);
                        if (prev == -1 || prev == nb[q]) {
                            slot = (int)h;
                            break;
                        }
                        h = (h + 1) & (kRedistTable - 1);
                    }
                    if (slot < 0) overflow = 1;
                }
                slots[(size_t)m * 7 + q] = (short)slot;
            }
        }
        __syncthreads();
        if (overflow) {  // the same in every thread: k_redist_par decides the list (a.cand is unchanged)
            if (threadIdx.x == 0) rs->par = 1;
            return;
        }
        for (int s = threadIdx.x; s < kRedistTable; s += blockDim.x) {
            int c = tkey[s];
            if (c >= 0) {
                tcnt[s] = a.count[c];
                tcav[s] = a.cavity[c];
            }
        }
    }
    __syncthreads();
    // ---- decisions. The reference's loop (solver.rs:476-555) in index order,
    // replayed in parallel rounds (the rule of k_redist_par below, on the
    // shared-memory table): every pending candidate claims its cell's slot and
    // the slots of its neighbours below the cap with a stamp ordering lower
    // indices first, and runs once it holds all of them. The cells such
    // candidates touch are disjoint, so the moves are the sequential ones.
    // Candidates crowded into a few cells (a fresh jet) decide about one per
    // cell and round: once a round decides fewer than kRoundsMinDecided,
    // thread 0 decides the pending rest in index order (below). Every
    // candidate decided in a round held its cells against all lower pending
    // ones, so the rest in index order sees the counts the sequential loop sees.
    const uint32_t cap = a.cap;
    bool finish_serial = !a.rounds;
    if (a.rounds) {
        for (uint32_t round = 1;; ++round) {
            const unsigned long long stamp = (unsigned long long)round << 32;
            const int rb = (int)(round & 1u);
            uint32_t dec = 0;
            for (uint32_t m = threadIdx.x; m < nc; m += blockDim.x) {
                const uint32_t p = scand[m];
                if (p & kResolved) continue;
                const short* sl = slots + (size_t)m * 7;
                const int s0 = sl[0];
                if (tcnt[s0] <= cap) {  // back at the cap: stays there for this sweep
                    scand[m] = p | kResolved;
                    ++dec;
                    continue;
                }
                const unsigned long long key = stamp | (unsigned long long)(0xFFFFFFFFu - m);
                bool any = false;
#pragma unroll
                for (int q = 1; q < 7; ++q) {
                    const int sq = sl[q];
                    if (sq >= 0 && tcav[sq] && tcnt[sq] < cap) {
                        atomicMax(tclaim + sq, key);
                        any = true;
                    }
                }
                if (!any) {  // no neighbour with room now, none later
                    scand[m] = p | kResolved;
                    ++dec;
                    continue;
                }
                atomicMax(tclaim + s0, key);
            }
            __syncthreads();
            if (threadIdx.x == 0) s_dec[rb ^ 1] = 0;  // every thread read it before the barrier above
            int pend = 0;
            for (uint32_t m = threadIdx.x; m < nc; m += blockDim.x) {
                const uint32_t p = scand[m];
                if (p & kResolved) continue;
                const short* sl = slots + (size_t)m * 7;
                const int s0 = sl[0];
                const unsigned long long key = stamp | (unsigned long long)(0xFFFFFFFFu - m);
                bool ready = tclaim[s0] == key;
                uint32_t cnt[6];
#pragma unroll
                for (int q = 1; q < 7; ++q) {
                    const int sq = sl[q];
                    cnt[q - 1] = (sq >= 0 && tcav[sq]) ? tcnt[sq] : 0xFFFFFFFFu;
                    if (cnt[q - 1] < cap && tclaim[sq] != key) ready = false;
                }
                if (!ready) {
                    pend = 1;
                    continue;
                }
                int best = -1;
                double best_down = -INFINITY;
                uint32_t best_room = 0;
#pragma unroll
                for (int q = 1; q < 7; ++q) {  // most downhill, then emptiest, then visit order
                    if (cnt[q - 1] >= cap) continue;
                    const uint32_t room = cap - cnt[q - 1];
                    const double dn = a.down[q - 1];
                    if (best < 0 || dn > best_down || (dn == best_down && room > best_room)) {
                        best = sl[q];
                        best_down = dn;
                        best_room = room;
                    }
                }
                scand[m] = p | kResolved;
                ++dec;
                if (best < 0) continue;  // its last neighbour with room was filled this round by a lower candidate
                tcnt[s0] -= 1;
                tcnt[best] += 1;
                const uint32_t slot = atomicAdd(&s_nm, 1u);
                a.moves[2 * slot] = p;
                a.moves[2 * slot + 1] = (uint32_t)tkey[best];
            }
            if (dec) atomicAdd(&s_dec[rb], dec);
            if (__syncthreads_count(pend) == 0) break;
            if (s_dec[rb] < kRoundsMinDecided) {  // the same value in every thread
                finish_serial = true;
                break;
            }
            if (round > nc) {  // cannot happen: the lowest pending candidate always runs
                if (threadIdx.x == 0) atomicOr(&rs->err, 4u);
                break;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        uint32_t nm = s_nm;
        if (finish_serial) {
            // One thread in index order over the candidates no round decided
            // (all of them without rounds): cheaper than rounds when a few
            // cells hold most candidates (a fresh jet), whose moves can only
            // run one per round; the moves are the same.
            for (uint32_t m = 0; m < nc; ++m) {
                if (cl[m] & kResolved) continue;
                const short* sl = slots + (size_t)m * 7;
                const int s0 = sl[0];
                if (tcnt[s0] <= cap) continue;
                int best = -1;
                double best_down = -INFINITY;
                uint32_t best_room = 0;
#pragma unroll
                for (int q = 1; q < 7; ++q) {
                    const int sq = sl[q];
                    if (sq < 0 || !tcav[sq] || tcnt[sq] >= cap) continue;
                    const uint32_t room = cap - tcnt[sq];
                    const double dn = a.down[q - 1];
                    if (best < 0 || dn > best_down || (dn == best_down && room > best_room)) {
                        best = sq;
                        best_down = dn;
                        best_room = room;
                    }
                }
                if (best >= 0) {
                    tcnt[s0] -= 1;
                    tcnt[best] += 1;
                    a.moves[2 * nm] = cl[m];
                    a.moves[2 * nm + 1] = (uint32_t)tkey[best];
                    ++nm;
                }
            }
        }
        s_nm = nm;
        rs->nmoves = nm;
        rs->moves_total += nm;
        rs->cand_total += nc;
        rs->sweeps_total += 1;
        rs->long_total += in_smem ? 0 : 1;
        rs->ncand = 0;
        if (nm == 0) rs->active = 0;
    }
    __syncthreads();
    // ---- apply the moves: near the destination centre with the index-keyed
    // jitter, pushed inside, with the local grid velocity.
    const uint32_t nm = s_nm;
    for (uint32_t mv = threadIdx.x; mv < nm; mv += blockDim.x) redist_apply_move(a, a.moves[2 * mv], a.moves[2 * mv + 1]);
}
__global__ void __launch_bounds__(kRedistBS, 1) k_redist_replay(RedistArgs a) { k_redist_replay_body(VB{blockIdx.x, gridDim.x}, a); }

constexpr size_t kRedistSmem = (size_t)kRedistTable * 8 + (size_t)kRedistTable * 4 * 2 +
                               (size_t)kRedistSmemCand * 4 + (size_t)kRedistSmemCand * 7 * 2 + kRedistTable;

// ---------------------------------------------------------------------------
// Long candidate lists: the reference's sequential loop (solver.rs:476-555)
// replayed in parallel rounds on one thread-block cluster, with the same moves.
//
// Within a sweep a cell only receives while below the cap and a source cell
// (above the cap) only loses particles and never drops below the cap. So a
// candidate's decision reads just two kinds of changing counts: its own cell's
// (changed only by candidates of that cell) and those of its neighbours that
// are below the cap (changed only by candidates that may choose them); every
// other neighbour is full or outside the cavity for the rest of the sweep.
// Each round every pending candidate m claims its cell and each neighbour
// still below the cap with a stamp that orders lower particle indices first;
// m runs when it holds all its claims, i.e. when no lower pending candidate
// can change what m reads or read what m changes. Those candidates run at
// once (their cells are disjoint), which is the sequential result. Candidates
// whose cell is back at the cap, or whose neighbours are all full, can never
// move again and leave the list. The lowest pending candidate always runs, so
// the rounds end; a bound on them still records an error bit if they did not.
// The long-list form (redist_par_run) decides units of one cell's consecutive
// candidates the same way.
constexpr int kRpBS = 512;
constexpr uint32_t kRpSoloList = 4 * kRpBS;  // pending units CTA 0 decides alone on the grid form

// The CTAs that decide one long list: one thread-block cluster (barrier in
// hardware), or every CTA of a cooperative launch (a bounded grid barrier;
// false if it gave up, with an error bit set).
struct RpCluster {
    static constexpr bool kGrid = false;
    __device__ int rank() const { return (int)cluster_rank(); }
    __device__ int size() const { return (int)cluster_size(); }
    __device__ bool sync() const {
        cluster_sync_all();
        return true;
    }
    double* slots;  // 2 x 16
};
struct RpGrid {
    static constexpr bool kGrid = true;
    __device__ int rank() const { return (int)blockIdx.x; }
    __device__ int size() const { return (int)gridDim.x; }
    __device__ bool sync() const { return grid_sync_bounded(bar, err, kErrGridWait); }
    double* slots;  // 2 x gridDim.x
    unsigned* bar;  // [0] arrivals, [1] generation
    uint32_t* err;
};

template <class Team>
__device__ void redist_par_run(const RedistArgs& a, const Team& team) {
    RedistState* rs = a.rs;
    if (!rs->active || !rs->par) return;  // written by earlier launches: the same in every CTA
    const int rank = team.rank(), nct = team.size();
    bool ok = true;
    const uint32_t gt = (uint32_t)(rank * kRpBS + threadIdx.x), G = (uint32_t)(nct * kRpBS);
    const uint32_t nc = rs->ncand, cap = a.cap;
    const Grid& g = a.g;
    const int sxy = g.nx * g.ny;
    uint32_t base = rs->round_base;
    if (rank == 0 && threadIdx.x == 0) rs->pend_n[0] = rs->pend_n[1] = 0u;
    ok = team.sync() && ok;  // every CTA has read the state before it changes
    if (base > 0xF0000000u) {  // stamps about to wrap: clear the claims and start again
        const size_t nce = (size_t)g.nx * g.ny * g.nz;
        for (size_t c = gt; c < nce; c += G) a.claim[c] = 0ull;
        base = 0;
        ok = team.sync() && ok;
    }
    // ---- the list in particle-index order: a bitmap of the candidates'
    // indices (distinct), counted per CTA chunk of words, then each CTA writes
    // its chunk's indices in order at its offset, over the list in place
    const uint32_t nw = (a.n_upper + 31u) / 32u;
    for (uint32_t w = gt; w < nw; w += G) a.bits[w] = 0u;
    ok = team.sync() && ok;
    for (uint32_t q = gt; q < nc; q += G) {
        const uint32_t p = a.cand[q];
        atomicOr(a.bits + (p >> 5), 1u << (p & 31u));
    }
    ok = team.sync() && ok;
    __shared__ uint32_t s_scan[kRpBS / 32 + 1];
    const uint32_t per = (nw + (uint32_t)nct - 1u) / (uint32_t)nct;
    const uint32_t w0 = min((uint32_t)rank * per, nw), w1 = min(w0 + per, nw);
    const uint32_t sub = (w1 - w0 + kRpBS - 1u) / kRpBS;  // words of this thread, contiguous
    const uint32_t tw0 = min(w0 + threadIdx.x * sub, w1), tw1 = min(tw0 + sub, w1);
    uint32_t mine = 0;
    for (uint32_t w = tw0; w < tw1; ++w) mine += __popc(__ldcg(a.bits + w));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t incl = mine;  // inclusive scan of this CTA's thread counts
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_scan[wid] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int w = 0; w < kRpBS / 32; ++w) {
            const uint32_t x = s_scan[w];
            s_scan[w] = run;
            run += x;
        }
        s_scan[kRpBS / 32] = run;  // this CTA's count
        team.slots[rank] = (double)run;  // exact: counts are below 2^32
    }
    __syncthreads();
    uint32_t at = s_scan[wid] + incl - mine;  // this thread's first position within the CTA
    ok = team.sync() && ok;
    if (threadIdx.x < 32) {  // this CTA's offset: the counts of the CTAs before it
        double off = 0.0;
        for (int r = lane; r < rank; r += 32) off += __ldcg(team.slots + r);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) off += __shfl_xor_sync(0xffffffffu, off, o);
        if (lane == 0) s_scan[kRpBS / 32] = (uint32_t)off;
    }
    __syncthreads();
    at += s_scan[kRpBS / 32];
    for (uint32_t w = tw0; w < tw1; ++w) {
        uint32_t b = __ldcg(a.bits + w);
        while (b) {
            const int k = __ffs((int)b) - 1;
            if (at < nc) a.cand[at] = w * 32u + (uint32_t)k;
            ++at;
            b &= b - 1u;
        }
    }
    ok = team.sync() && ok;
    // ---- units: a maximal run of consecutive candidates (index order) in one
    // cell. The reference's loop (solver.rs:476-555) takes a run's candidates
    // one after another with no other candidate between them, so a unit is
    // decided as one: it claims its cell and its neighbours below the cap with
    // a stamp that orders lower heads first, and once it holds every claim one
    // thread takes its candidates in index order (the moves are the
    // sequential ones: no lower pending unit reads or changes those cells).
    // The first round's list is every unit's head position.
    uint32_t* pb = a.pend;
    for (uint32_t q = gt; q < nc; q += G) {
        const int c = a.key_cell[a.cand[q]];
        if (q == 0 || a.key_cell[a.cand[q - 1]] != c) pb[atomicAdd(&rs->pend_n[0], 1u)] = q;
    }
    ok = team.sync() && ok;
    // The units still pending after a round go to the other half of `pend`
    // (any order: a claim's stamp carries the head's index), so a round
    // touches only those. On the whole grid, once few remain CTA 0 decides
    // them alone (block barriers instead of grid barriers) while the others
    // wait at the barrier below.
    const uint32_t* pa = pb;
    pb = a.pend + a.cand_cap;
    uint32_t na = __ldcg(&rs->pend_n[0]);
    uint32_t round = 0;
    bool solo = false;
    uint32_t gt_ = gt, G_ = G;
    while (na > 0 && ok) {
        if (Team::kGrid && !solo && na <= kRpSoloList) {  // the same decision in every CTA
            solo = true;
            if (rank != 0) break;
            gt_ = threadIdx.x;
            G_ = kRpBS;
        }
        ++round;
        const int cur = (int)(round & 1u);
        const unsigned long long stamp = (unsigned long long)(base + round) << 32;
        // claims (or leave the list)
        for (uint32_t q = gt_; q < na; q += G_) {
            const uint32_t m = pa[q];
            const uint32_t p = a.cand[m];
            if (p & kResolved) continue;
            const int c = a.key_cell[p];
            if (__ldcg(a.count + c) <= cap) {
                a.cand[m] = p | kResolved;
                continue;
            }
            const int i = c % g.nx, j = (c / g.nx) % g.ny, k = c / sxy;
            const int nb[6] = {i > 0 ? c - 1 : -1, i + 1 < g.nx ? c + 1 : -1, j > 0 ? c - g.nx : -1,
                               j + 1 < g.ny ? c + g.nx : -1, k > 0 ? c - sxy : -1, k + 1 < g.nz ? c + sxy : -1};
            const unsigned long long key = stamp | (unsigned long long)(0xFFFFFFFFu - p);
            bool any = false;
#pragma unroll
            for (int qq = 0; qq < 6; ++qq) {
                const int n = nb[qq];
                if (n >= 0 && a.cavity[n] && __ldcg(a.count + n) < cap) {
                    atomicMax(a.claim + n, key);
                    any = true;
                }
            }
            if (!any) {
                a.cand[m] = p | kResolved;
                continue;
            }
            atomicMax(a.claim + c, key);
        }
        if (solo) __syncthreads();
        else ok = team.sync() && ok;
        // units holding all their claims run (counts are as in the claim
        // step); the others go on the next round's list
        for (uint32_t q = gt_; q < na; q += G_) {
            const uint32_t m = pa[q];
            const uint32_t p = a.cand[m];
            if (p & kResolved) continue;
            const int c = a.key_cell[p];
            const unsigned long long key = stamp | (unsigned long long)(0xFFFFFFFFu - p);
            const int i = c % g.nx, j = (c / g.nx) % g.ny, k = c / sxy;
            const int nb[6] = {i > 0 ? c - 1 : -1, i + 1 < g.nx ? c + 1 : -1, j > 0 ? c - g.nx : -1,
                               j + 1 < g.ny ? c + g.nx : -1, k > 0 ? c - sxy : -1, k + 1 < g.nz ? c + sxy : -1};
            bool ready = __ldcg(a.claim + c) == key;
#pragma unroll
            for (int qq = 0; qq < 6; ++qq) {
                const int n = nb[qq];
                if (n >= 0 && a.cavity[n] && __ldcg(a.count + n) < cap && __ldcg(a.claim + n) != key) ready = false;
            }
            if (!ready) {
                pb[atomicAdd(&rs->pend_n[cur], 1u)] = m;
                continue;
            }
            // The unit's candidates in index order, on its counts held in
            // registers (the unit holds its cell and every neighbour with room;
            // a full neighbour stays full within a sweep): each moves while the
            // cell is above the cap and a neighbour has room, so the first
            // min(excess, total room, unit length) move, to the neighbours the
            // reference's rule picks as the counts change.
            uint32_t cc = __ldcg(a.count + c);
            uint32_t cn[6];
            uint32_t room = 0;
#pragma unroll
            for (int qq = 0; qq < 6; ++qq) {
                const int n = nb[qq];
                cn[qq] = (n >= 0 && a.cavity[n]) ? __ldcg(a.count + n) : cap;  // outside: full
                if (cn[qq] < cap) room += cap - cn[qq];
            }
            const uint32_t need = min(cc > cap ? cc - cap : 0u, room);
            uint32_t nmov = need > 0 ? 1u : 0u;  // the head is a member
            while (nmov < need && m + nmov < nc && a.key_cell[a.cand[m + nmov] & ~kResolved] == c) ++nmov;
            if (nmov > 0) {
                const uint32_t slot0 = atomicAdd(&rs->nmoves_par, nmov);
                uint32_t moved = 0u;  // neighbours that received (bit per direction)
                for (uint32_t u = 0; u < nmov; ++u) {
                    int best = -1, best_n = -1;
                    double best_down = -INFINITY;
                    uint32_t best_room = 0;
#pragma unroll
                    for (int qq = 0; qq < 6; ++qq) {  // solver.rs:519-544: most downhill, then emptiest, then visit order
                        if (cn[qq] >= cap) continue;
                        const uint32_t rq = cap - cn[qq];
                        const double dn = a.down[qq];
                        if (best < 0 || dn > best_down || (dn == best_down && rq > best_room)) {
                            best = qq;
                            best_n = nb[qq];
                            best_down = dn;
                            best_room = rq;
                        }
                    }
                    if (best < 0) {  // cannot happen (each move takes one unit of the room counted above):
                        atomicOr(&rs->err, 4u);  // the reserved slot still gets a defined move
                        best_n = c;
                    } else {
#pragma unroll
                        for (int qq = 0; qq < 6; ++qq)
                            if (qq == best) cn[qq] += 1u;  // static indices keep cn in registers
                        moved |= 1u << best;
                    }
                    a.moves[2 * (slot0 + u)] = u == 0 ? p : (a.cand[m + u] & ~kResolved);
                    a.moves[2 * (slot0 + u) + 1] = (uint32_t)best_n;
                }
                a.count[c] = cc - nmov;
#pragma unroll
                for (int qq = 0; qq < 6; ++qq)
                    if (moved >> qq & 1u) a.count[nb[qq]] = cn[qq];
            }
            a.cand[m] = p | kResolved;
        }
        if (solo) __syncthreads();
        else ok = team.sync() && ok;
        na = __ldcg(&rs->pend_n[cur]);
        // the other counter was last read after the previous round: clear it
        // for the next round's appends (ordered before them by its first barrier)
        if (rank == 0 && threadIdx.x == 0) rs->pend_n[cur ^ 1] = 0u;
        pa = pb;
        pb = (pb == a.pend) ? a.pend + a.cand_cap : a.pend;
        if (na > 0 && round > nc) {  // cannot happen: the lowest pending unit always runs
            if (rank == 0 && threadIdx.x == 0) atomicOr(&rs->err, 4u);
            break;
        }
    }
    if (solo) ok = team.sync() && ok;  // CTA 0 arrives once its rounds are done
    const uint32_t nm = __ldcg(&rs->nmoves_par);
    for (uint32_t mv = gt; mv < nm; mv += G) redist_apply_move(a, a.moves[2 * mv], a.moves[2 * mv + 1]);
    ok = team.sync() && ok;
    if (rank == 0 && threadIdx.x == 0) {
        rs->nmoves = nm;
        rs->moves_total += nm;
        rs->cand_total += nc;
        rs->sweeps_total += 1;
        rs->long_total += 1;
        rs->ncand = 0;
        rs->par = 0;
        rs->nmoves_par = 0;
        rs->round_base = base + round + 1;
        rs->rounds_total += round;
        if (nm == 0) rs->active = 0;
    }
}
__device__ __forceinline__ void k_redist_par_body(VB, RedistArgs a) {
    RpCluster t;
    t.slots = a.slots;
    redist_par_run(a, t);
}
__global__ void __launch_bounds__(kRpBS, 1) k_redist_par(RedistArgs a) { k_redist_par_body(VB{blockIdx.x, gridDim.x}, a); }

// The same rounds over every SM: a cooperative launch, one CTA per team rank.
__global__ void __launch_bounds__(kRpBS, 2) k_redist_par_grid(RedistArgs a, double* slots, unsigned* bar) {
    RpGrid t;
    t.slots = slots;
    t.bar = bar;
    t.err = &a.rs->err;
    redist_par_run(a, t);
}

}  // namespace sdr
