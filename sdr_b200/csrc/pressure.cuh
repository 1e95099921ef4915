// Pressure projection (src/pressure.rs:123-609) on the device.
//
// Layout: fluid cells are numbered in wavefront order — by level L = i+j+k,
// and within a level by (k, j) — so that each MIC(0) triangular sweep is a
// walk over contiguous level ranges whose predecessors (-x,-y,-z) all sit in
// level L-1 and successors in level L+1. All PCG vectors are compact f64 in
// that order. The Laplacian is never stored: diag (non-solid neighbour
// count) and the neighbour table come from the labels (pressure.rs:170-223).
//
// Bit-exactness: every f64 operation is an explicit round-to-nearest
// intrinsic in the reference's order, the dot product reproduces its fixed
// 4096-cell chunking with in-chunk sequential sums (pressure.rs:588-603), and
// the MIC(0) factor/sweeps perform the same per-cell arithmetic as the
// sequential loops. Given the same labels and RHS, pressure and iteration
// count equal the CPU reference's bit for bit.
#pragma once
#include "common.cuh"
#include "particles.cuh"

namespace sdr {

constexpr int kDotChunk = 4096;
constexpr int kPcgBS = 768;
constexpr int kPcgWin = 6144;  // smem window (doubles) per level buffer

// Neighbour directions in the reference's visit order.
enum { NB_MX = 0, NB_PX = 1, NB_MY = 2, NB_PY = 3, NB_MZ = 4, NB_PZ = 5 };

// Count fluid cells on each (level, k) line: cells (i, j, k) with i + j + k = L.
__device__ __forceinline__ void k_lines_count_body(VB vb_, Grid g, const uint8_t* __restrict__ cells, int nlevels,
                              uint32_t* __restrict__ cnt) {
    int t = vb_.bid * blockDim.x + threadIdx.x;
    if (t >= nlevels * g.nz) return;
    int L = t / g.nz, k = t % g.nz;
    int r = L - k;  // i + j = r
    uint32_t n = 0;
    int j0 = max(0, r - (g.nx - 1)), j1 = min(g.ny - 1, r);
    for (int j = j0; j <= j1; ++j) {
        int i = r - j;
        n += cells[((size_t)k * g.ny + j) * g.nx + i] == FLUID;
    }
    cnt[t] = n;
}
__global__ void k_lines_count(Grid g, const uint8_t* __restrict__ cells, int nlevels,
                              uint32_t* __restrict__ cnt) { k_lines_count_body(VB{blockIdx.x, gridDim.x}, g, cells, nlevels, cnt); }

// Assign wavefront positions: pos = line base + rank along j.
__device__ __forceinline__ void k_lines_assign_body(VB vb_, Grid g, const uint8_t* __restrict__ cells, int nlevels,
                               const uint32_t* __restrict__ base, int* __restrict__ pos_of_cell,
                               uint32_t* __restrict__ lv_cell) {
    int t = vb_.bid * blockDim.x + threadIdx.x;
    if (t >= nlevels * g.nz) return;
    int L = t / g.nz, k = t % g.nz;
    int r = L - k;
    uint32_t pos = base[t];
    int j0 = max(0, r - (g.nx - 1)), j1 = min(g.ny - 1, r);
    for (int j = j0; j <= j1; ++j) {
        int i = r - j;
        size_t c = ((size_t)k * g.ny + j) * g.nx + i;
        if (cells[c] == FLUID) {
            pos_of_cell[c] = (int)pos;
            lv_cell[pos] = (uint32_t)c;
            ++pos;
        }
    }
}
__global__ void k_lines_assign(Grid g, const uint8_t* __restrict__ cells, int nlevels,
                               const uint32_t* __restrict__ base, int* __restrict__ pos_of_cell,
                               uint32_t* __restrict__ lv_cell) { k_lines_assign_body(VB{blockIdx.x, gridDim.x}, g, cells, nlevels, base, pos_of_cell, lv_cell); }

// Level starts from the (level, k) line bases; nf is the device fluid count.
__device__ __forceinline__ void k_level_starts_dev_body(VB vb_, const uint32_t* __restrict__ base, int nlevels, int nz,
                                   const uint32_t* __restrict__ nf, int* __restrict__ level_start) {
    int L = vb_.bid * blockDim.x + threadIdx.x;
    if (L < nlevels) level_start[L] = (int)base[L * nz];
    if (L == nlevels) level_start[L] = (int)*nf;
}
__global__ void k_level_starts_dev(const uint32_t* __restrict__ base, int nlevels, int nz,
                                   const uint32_t* __restrict__ nf, int* __restrict__ level_start) { k_level_starts_dev_body(VB{blockIdx.x, gridDim.x}, base, nlevels, nz, nf, level_start); }

struct TableArgs {
    Grid g;
    const uint8_t* cells;
    const int* pos_of_cell;
    const uint32_t* lv_cell;
    const uint32_t* nf;  // device fluid count
    int* nbr;          // 6 per fluid cell (compact position or -1)
    uint8_t* diag;     // non-solid in-bounds neighbours (pressure.rs:187-220)
    uint8_t* nmask;    // bit d: neighbour d is fluid
    double* b;         // RHS (pressure.rs:152-168)
    const float* u;
    const float* v;
    const float* w;
    const uint32_t* hist;  // particles per cell (for the volume source)
    double inv_scale;      // rho*dx/dt
    // volume source (solver.rs:392-423)
    int vs_on;
    double vs_rest, vs_k, vs_unit, vs_cap;
};

// Per fluid cell: neighbour table, diag, and the RHS b = -(rho dx/dt)(div - s).
__device__ __forceinline__ void k_tables_body(VB vb_, TableArgs a) {
    uint32_t pos = vb_.bid * blockDim.x + threadIdx.x;
    if (pos >= *a.nf) return;
    const Grid& g = a.g;
    uint32_t c = a.lv_cell[pos];
    int i = c % g.nx, j = (c / g.nx) % g.ny, k = c / (g.nx * g.ny);
    int nb[6];
    uint8_t diag = 0, mask = 0;
    const int off[6] = {-1, 1, -g.nx, g.nx, -g.nx * g.ny, g.nx * g.ny};
    const bool inb[6] = {i > 0, i + 1 < g.nx, j > 0, j + 1 < g.ny, k > 0, k + 1 < g.nz};
    for (int d = 0; d < 6; ++d) {
        nb[d] = -1;
        if (!inb[d]) continue;
        uint32_t nc = c + off[d];
        uint8_t lab = a.cells[nc];
        if (lab != SOLID) ++diag;
        if (lab == FLUID) {
            nb[d] = a.pos_of_cell[nc];
            mask |= (uint8_t)(1u << d);
        }
    }
#pragma unroll
    for (int d = 0; d < 6; ++d) a.nbr[(size_t)pos * 6 + d] = nb[d];
    a.diag[pos] = diag;
    a.nmask[pos] = mask;
    // divergence from f32 faces in f64 (pressure.rs:161-163)
    size_t ui = ((size_t)k * g.ny + j) * (g.nx + 1) + i;
    size_t vi = ((size_t)k * (g.ny + 1) + j) * g.nx + i;
    size_t wi = ((size_t)k * g.ny + j) * g.nx + i;
    double du = dsub((double)a.u[ui + 1], (double)a.u[ui]);
    double dv = dsub((double)a.v[vi + g.nx], (double)a.v[vi]);
    double dw = dsub((double)a.w[wi + (size_t)g.nx * g.ny], (double)a.w[wi]);
    double div = dadd(dadd(du, dv), dw);
    double s = 0.0;
    if (a.vs_on) {
        double over = dsub(ddiv((double)a.hist[c], a.vs_rest), 1.0);
        if (over > 0.0) s = fmin(dmul(dmul(a.vs_k, over), a.vs_unit), a.vs_cap);
    }
    a.b[pos] = dmul(-a.inv_scale, dsub(div, s));
}
__global__ void k_tables(TableArgs a) { k_tables_body(VB{blockIdx.x, gridDim.x}, a); }

// Fluid cells in cell-index order -> wavefront position, for the chunked dot.
__device__ __forceinline__ void k_fluid_flags_body(VB vb_, const uint8_t* __restrict__ cells, size_t n, uint32_t* __restrict__ flag) {
    size_t c = (size_t)vb_.bid * blockDim.x + threadIdx.x;
    if (c < n) flag[c] = cells[c] == FLUID;
}
__global__ void k_fluid_flags(const uint8_t* __restrict__ cells, size_t n, uint32_t* __restrict__ flag) { k_fluid_flags_body(VB{blockIdx.x, gridDim.x}, cells, n, flag); }

__device__ __forceinline__ void k_corder_body(VB vb_, const uint8_t* __restrict__ cells, size_t n, const uint32_t* __restrict__ off,
                         const int* __restrict__ pos_of_cell, int* __restrict__ corder, int* __restrict__ cinv,
                         int* __restrict__ chunk_start, int nchunks, const uint32_t* __restrict__ nf) {
    size_t c = (size_t)vb_.bid * blockDim.x + threadIdx.x;
    if (c < n && cells[c] == FLUID) {
        corder[off[c]] = pos_of_cell[c];
        cinv[pos_of_cell[c]] = (int)off[c];
    }
    if (c < n && c % kDotChunk == 0) chunk_start[c / kDotChunk] = (int)off[c];
    if (c == 0) chunk_start[nchunks] = (int)*nf;
}
__global__ void k_corder(const uint8_t* __restrict__ cells, size_t n, const uint32_t* __restrict__ off,
                         const int* __restrict__ pos_of_cell, int* __restrict__ corder, int* __restrict__ cinv,
                         int* __restrict__ chunk_start, int nchunks, const uint32_t* __restrict__ nf) { k_corder_body(VB{blockIdx.x, gridDim.x}, cells, n, off, pos_of_cell, corder, cinv, chunk_start, nchunks, nf); }

struct PcgArgs {
    const uint32_t* nf;  // device fluid count
    int nlevels;
    int nchunks;
    int nx, ny;
    const int* level_start;
    const int* nbr;
    const uint8_t* diag;
    const uint8_t* nmask;
    const int* corder;
    const int* cinv;        // wavefront position -> cell-order index
    const int* chunk_start;
    const double* b;
    double* precon;
    double* p;
    double* r;
    double* z;
    double* s;
    double* as;
    double* q;
    double* pq;
    double* prod;       // per-cell products: cell order (reference dots) or wavefront order (tree dots)
    double* partials;   // nchunks: reference-order chunk sums
    double* tpart;      // ceil(nf / kTile): tree-order tile sums
    double* slots;      // 2 x 16: CTA partials of cluster-wide maxima
    int4* frec;         // per cell: forward sweep record (precon + window slots of -x,-y,-z)
    int4* brec;         // per cell: backward sweep record (precon + window slots of +x,+y,+z)
    double tol;
    int max_iters;
    const uint32_t* lv_cell;
    double* p_dense;    // pre-zeroed; fluid cells written at exit
    int* out_iters;
    double* out_residual;
    unsigned long long* timing;  // optional: cycles per section
    int exact_dots;              // 1: the reference's chunked sequential dot order (bit-exact); 0: fixed block tree
};

// Sweep record: the cell's MIC factor and the shared-window slots (index
// within the neighbouring level, -1 = not fluid) of its three neighbours.
struct SweepRec {
    double pc;
    short s0, s1, s2, pad;
};

// Shared-memory plan of k_pcg (dynamic): a ring of kStages staged levels
// (two f64 operands and one record per cell), two level windows of f64 and of
// neighbour masks and the level starts.
constexpr int kStages = 4;          // levels in flight ahead of the sweep
constexpr int kMaxLevelsSmem = 2048;
constexpr int kSweepMax = kPcgBS - 32;  // compute threads; one producer warp stages ahead
constexpr size_t kPcgSmem = (size_t)kStages * kPcgBS * (8 + 8 + 16) + 2 * kPcgBS * 8 + 2 * kPcgBS * 4 +
                            (kMaxLevelsSmem + 1) * 4;

struct PcgSmem {
    double* sa;     // [kStages][BS]
    double* sb;     // [kStages][BS]
    SweepRec* sr;   // [kStages][BS]
    double* w0;     // [BS] level window
    double* w1;
    int* m0;        // [BS] neighbour-mask window (MIC build)
    int* m1;
    int* lvs;       // level starts (smem copy or global)
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// The producer keeps two levels complete ahead of the one being computed, so
// compute threads can read level L+1's staged data into registers while level
// L is in flight.
__device__ __forceinline__ void cp_wait_ahead() {
    asm volatile("cp.async.wait_group %0;" ::"n"(kStages - 3) : "memory");
}

// Barrier over the first `n` threads (named barrier 1): the sweeps run on the
// compute warps plus one producer warp, sized to the widest level, so the
// per-level barrier carries only working warps.
__device__ __forceinline__ void sweep_bar(int n) { asm volatile("bar.sync 1, %0;" ::"r"(n) : "memory"); }

// Producer warp: stage every cell of level L (if the level fits the ring)
// into slot L % kStages: operand A, optional operand B, and the record.
__device__ __forceinline__ void produce_level(const PcgSmem& m, int L, int lo, int hi, const double* va,
                                              const double* vb, const int4* rec, int lane) {
    if (L >= lo && L < hi) {
        int ls = m.lvs[L], le = m.lvs[L + 1];
        if (le - ls <= kSweepMax) {
            int base = (L % kStages) * kPcgBS;
            for (int t = lane; t < le - ls; t += 32) {
                cp_async8(&m.sa[base + t], &va[ls + t]);
                if (vb) cp_async8(&m.sb[base + t], &vb[ls + t]);
                cp_async16(&m.sr[base + t], &rec[ls + t]);
            }
        }
    }
    cp_commit();
}

// ---------------------------------------------------------------- cluster pieces
// The solve kernels run as one thread-block cluster (k_pcg: 1 CTA when the
// GPU is shared with other scenes, else up to 16; k_pcg_cluster: 16). These
// helpers split elementwise work and reductions over every thread of the
// cluster; a cluster barrier (hardware, release/acquire) orders the phases,
// and values another CTA wrote are read through L2.
constexpr int kTile = 256;      // cells per tile of the tree-order dot (wavefront order)
constexpr int kMaxCtas = 16;

struct PcgCl {
    int rank, nct;
    uint32_t gt, G;  // thread index and count over the cluster
    int gw, nw;      // warp index and count over the cluster
    int parity;      // half of `slots` the next maximum uses
};

__device__ __forceinline__ PcgCl pcg_cl() {
    PcgCl c;
    c.rank = (int)cluster_rank();
    c.nct = (int)cluster_size();
    c.gt = (uint32_t)c.rank * blockDim.x + threadIdx.x;
    c.G = (uint32_t)c.nct * blockDim.x;
    c.gw = c.rank * (int)(blockDim.x >> 5) + (int)(threadIdx.x >> 5);
    c.nw = c.nct * (int)(blockDim.x >> 5);
    c.parity = 0;
    return c;
}

__device__ __forceinline__ double warp_tree_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = dadd(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;  // the same bits in every lane (each step adds the same pair)
}

// Maximum over the cluster (order-free): per-CTA block maxima through a
// double-buffered slot array; a barrier separates a use of one half from the
// next use of the same half.
template <int BS>
__device__ __forceinline__ double pcg_cl_max(PcgCl& c, const PcgArgs& a, double v, double* sh) {
    double bm = block_max<BS>(v, sh);
    double* sl = a.slots + c.parity * kMaxCtas;
    c.parity ^= 1;
    if (threadIdx.x == 0) sl[c.rank] = bm;
    cluster_sync_all();
    double m = 0.0;
    for (int q = 0; q < c.nct; ++q) m = fmax(m, __ldcg(sl + q));
    return m;
}

// Tree-order dot (the default). Cells in wavefront order form tiles of
// kTile; lane l of the warp that owns a tile adds its cells l, l+32, ... in
// order and a fixed xor tree adds the 32 lanes; the tile sums are added the
// same way (lane l: tiles l, l+32, ...). The order depends on neither the
// number of CTAs nor the kernel, so every solve kernel gives the same bits.
__device__ __forceinline__ double pcg_tile_total(const PcgArgs& a, uint32_t ntile) {
    double s = 0.0;
    for (uint32_t t = threadIdx.x & 31; t < ntile; t += 32) s = dadd(s, __ldcg(a.tpart + t));
    return warp_tree_sum(s);
}

__device__ __forceinline__ double pcg_tree_dot_prod(const PcgArgs& a, const PcgCl& c, uint32_t nf) {
    cluster_sync_all();  // products complete
    const int lane = threadIdx.x & 31;
    const uint32_t ntile = (nf + kTile - 1) / kTile;
    for (uint32_t t = (uint32_t)c.gw; t < ntile; t += (uint32_t)c.nw) {
        double s = 0.0;
        const uint32_t e = min((t + 1) * kTile, nf);
        for (uint32_t i = t * kTile + lane; i < e; i += 32) s = dadd(s, __ldcg(a.prod + i));
        s = warp_tree_sum(s);
        if (lane == 0) a.tpart[t] = s;
    }
    cluster_sync_all();
    return pcg_tile_total(a, ntile);
}

// Exact reference dot (pressure.rs:588-603) over `prod` (cell order): one
// warp per 4096-cell chunk across the cluster folds its products in cell
// order, then every CTA adds the chunk sums in chunk order.
__device__ double pcg_exact_dot(const PcgArgs& a, const PcgCl& c, double* sh) {
    cluster_sync_all();  // products complete
    const int lane = threadIdx.x & 31;
    for (int ch = c.gw; ch < a.nchunks; ch += c.nw) {
        int t = a.chunk_start[ch], e = a.chunk_start[ch + 1];
        double acc = 0.0;
        for (; t < e; t += 512) {
            double v[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) {
                int idx = t + u * 32 + lane;
                v[u] = idx < e ? __ldcg(a.prod + idx) : 0.0;
            }
            int cnt = min(512, e - t);
#pragma unroll
            for (int u = 0; u < 16; ++u) {
#pragma unroll 8
                for (int src = 0; src < 32; ++src) {
                    double x = __shfl_sync(0xffffffffu, v[u], src);
                    if (u * 32 + src < cnt) acc = dadd(acc, x);
                }
            }
        }
        if (lane == 0) a.partials[ch] = acc;
    }
    cluster_sync_all();
    if (threadIdx.x == 0) {
        double s = -0.0;
        for (int ch = 0; ch < a.nchunks; ++ch) s = dadd(s, __ldcg(a.partials + ch));
        sh[0] = s;
    }
    __syncthreads();
    double r = sh[0];
    __syncthreads();
    return r;
}

// dot over the products a sweep or the matvec stored in `prod`.
__device__ __forceinline__ double pcg_dot_prod(const PcgArgs& a, const PcgCl& c, uint32_t nf, double* sh) {
    return a.exact_dots ? pcg_exact_dot(a, c, sh) : pcg_tree_dot_prod(a, c, nf);
}

// Tree dot of the products one CTA stored itself (the sweeps): that CTA forms
// the tile sums (same tiles and order as pcg_tree_dot_prod) and one cluster
// barrier publishes them. Called by every CTA; only `owner` does the tiles.
__device__ __forceinline__ double pcg_tree_dot_own(const PcgArgs& a, bool owner, uint32_t nf) {
    const uint32_t ntile = (nf + kTile - 1) / kTile;
    if (owner) {
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
        for (uint32_t t = w; t < ntile; t += nw) {
            double s = 0.0;
            const uint32_t e = min((t + 1) * kTile, nf);
            for (uint32_t i = t * kTile + lane; i < e; i += 32) s = dadd(s, a.prod[i]);
            s = warp_tree_sum(s);
            if (lane == 0) a.tpart[t] = s;
        }
    }
    cluster_sync_all();
    return pcg_tile_total(a, ntile);
}

// build_mic0 (pressure.rs:442-513) as a forward level sweep. precon and the
// neighbour mask of level L-1 come from the shared windows.
__device__ void pcg_build_mic0(const PcgArgs& a, const PcgSmem& m, int sw, int l0, int l1) {
    const double TAU = 0.97, SIGMA = 0.25;
    if ((int)threadIdx.x >= sw) {
        __syncthreads();
        return;
    }
    double* prev = m.w0;
    double* cur = m.w1;
    int* mprev = m.m0;
    int* mcur = m.m1;
    for (int L = l0; L < l1; ++L) {
        int ls = m.lvs[L], le = m.lvs[L + 1];
        int lsp = L > 0 ? m.lvs[L - 1] : 0;
        bool prev_in = L > l0 && (ls - lsp) <= kPcgBS;
        bool cur_in = (le - ls) <= kPcgBS;
        for (int ps = ls + threadIdx.x; ps < le; ps += sw) {
            const int* nb = a.nbr + (size_t)ps * 6;
            double axi = 0, pxi = 0, axi_y = 0, axi_z = 0;
            double ayj = 0, pyj = 0, ayj_x = 0, ayj_z = 0;
            double azk = 0, pzk = 0, azk_x = 0, azk_y = 0;
            int mm = nb[NB_MX];
            if (mm >= 0) {
                int mk = prev_in ? mprev[mm - lsp] : a.nmask[mm];
                axi = -1.0;
                pxi = prev_in ? prev[mm - lsp] : a.precon[mm];
                axi_y = (mk >> NB_PY & 1) ? -1.0 : 0.0;
                axi_z = (mk >> NB_PZ & 1) ? -1.0 : 0.0;
            }
            mm = nb[NB_MY];
            if (mm >= 0) {
                int mk = prev_in ? mprev[mm - lsp] : a.nmask[mm];
                ayj = -1.0;
                pyj = prev_in ? prev[mm - lsp] : a.precon[mm];
                ayj_x = (mk >> NB_PX & 1) ? -1.0 : 0.0;
                ayj_z = (mk >> NB_PZ & 1) ? -1.0 : 0.0;
            }
            mm = nb[NB_MZ];
            if (mm >= 0) {
                int mk = prev_in ? mprev[mm - lsp] : a.nmask[mm];
                azk = -1.0;
                pzk = prev_in ? prev[mm - lsp] : a.precon[mm];
                azk_x = (mk >> NB_PX & 1) ? -1.0 : 0.0;
                azk_y = (mk >> NB_PY & 1) ? -1.0 : 0.0;
            }
            double tx = dmul(axi, pxi), ty = dmul(ayj, pyj), tz = dmul(azk, pzk);
            double diag = (double)a.diag[ps];
            double mx = dmul(dmul(dmul(axi, dadd(axi_y, axi_z)), pxi), pxi);
            double my = dmul(dmul(dmul(ayj, dadd(ayj_x, ayj_z)), pyj), pyj);
            double mz = dmul(dmul(dmul(azk, dadd(azk_x, azk_y)), pzk), pzk);
            double e = dsub(dsub(dsub(dsub(diag, dmul(tx, tx)), dmul(ty, ty)), dmul(tz, tz)),
                            dmul(TAU, dadd(dadd(mx, my), mz)));
            if (e < dmul(SIGMA, diag)) e = diag;
            double pc = e > 0.0 ? ddiv(1.0, __dsqrt_rn(e)) : 0.0;
            a.precon[ps] = pc;
            if (cur_in) {
                cur[ps - ls] = pc;
                mcur[ps - ls] = a.nmask[ps];
            }
        }
        sweep_bar(sw);
        double* t = prev;
        prev = cur;
        cur = t;
        int* tm = mprev;
        mprev = mcur;
        mcur = tm;
    }
    __syncthreads();
}

// Per-solve sweep records from the neighbour table and the factor.
__device__ void pcg_build_records(const PcgArgs& a, const PcgSmem& m, uint32_t nf) {
    for (uint32_t ps = threadIdx.x; ps < nf; ps += blockDim.x) {
        uint32_t c = a.lv_cell[ps];
        int i = c % a.nx, j = (c / a.nx) % a.ny, k = c / (a.nx * a.ny);
        int L = i + j + k;
        const int* nb = a.nbr + (size_t)ps * 6;
        int lsp = L > 0 ? m.lvs[L - 1] : 0, lsn = m.lvs[L + 1];
        SweepRec f, g;
        f.pc = g.pc = a.precon[ps];
        int mm;
        f.s0 = (short)((mm = nb[NB_MX]) >= 0 ? mm - lsp : -1);
        f.s1 = (short)((mm = nb[NB_MY]) >= 0 ? mm - lsp : -1);
        f.s2 = (short)((mm = nb[NB_MZ]) >= 0 ? mm - lsp : -1);
        g.s0 = (short)((mm = nb[NB_PX]) >= 0 ? mm - lsn : -1);
        g.s1 = (short)((mm = nb[NB_PY]) >= 0 ? mm - lsn : -1);
        g.s2 = (short)((mm = nb[NB_PZ]) >= 0 ? mm - lsn : -1);
        f.pad = g.pad = 0;
        a.frec[ps] = *reinterpret_cast<int4*>(&f);
        a.brec[ps] = *reinterpret_cast<int4*>(&g);
    }
    __syncthreads();
}

// apply_mic0 (pressure.rs:517-570): forward L q = r then backward L^T z = q.
// Forward:  t = r + pq[-x] + pq[-y] + pq[-z]  (pq = precon*q of the predecessor,
//           which is what `t -= plus*precon*q` with plus = -1 adds), q = t*pc.
// Backward: t = q + pc*z[+x] + pc*z[+y] + pc*z[+z], z = t*pc, plus the z*r
//           products of the following dot.
// Compute threads [0, sw) take one cell each per level from the staged ring;
// the producer warp [sw, sw+32) stages level L + kStages - 1 while level L is
// computed. Levels wider than the ring use global memory (uniform branch).
__device__ void pcg_apply_mic0(const PcgArgs& a, const PcgSmem& m, const double* r, double* z, int sw, int l0,
                               int l1, unsigned long long* lt = nullptr) {
    const int tid = threadIdx.x;
    const int nbar = sw + 32;
    if (tid >= nbar) {
        __syncthreads();
        return;
    }
    const bool producer = tid >= sw;
    const int lane = tid - sw;
    // ---------------- forward
    if (producer) {
        for (int d = 0; d < kStages - 1; ++d) produce_level(m, l0 + d, l0, l1, r, nullptr, a.frec, lane);
        cp_wait_ahead();
    }
    sweep_bar(nbar);
    double* prev = m.w0;
    double* cur = m.w1;
    int lsP = l0 > 0 ? m.lvs[l0 - 1] : 0, lsA = m.lvs[l0], lsB = m.lvs[l0 + 1];
    // staged operands of this thread's cell in the current level (registers)
    double ct = 0.0;
    SweepRec crc{};
    if (!producer && tid < lsB - lsA && lsB - lsA <= kSweepMax) {
        int slot = (l0 % kStages) * kPcgBS + tid;
        ct = m.sa[slot];
        crc = m.sr[slot];
    }
    for (int L = l0; L < l1; ++L) {
        int lsC = m.lvs[min(L + 2, a.nlevels)];
        unsigned long long c0 = lt ? clock64() : 0;
        const int wprev = lsA - lsP, wcur = lsB - lsA, wnext = lsC - lsB;
        double nt_ = 0.0;
        SweepRec nrc{};
        if (producer) {
            produce_level(m, L + kStages - 1, l0, l1, r, nullptr, a.frec, lane);
            cp_wait_ahead();
        } else {
            if (L + 1 < l1 && tid < wnext && wnext <= kSweepMax) {  // prefetch level L+1
                int slot = ((L + 1) % kStages) * kPcgBS + tid;
                nt_ = m.sa[slot];
                nrc = m.sr[slot];
            }
            if (wcur <= kSweepMax) {
                if (tid < wcur) {
                    double t = ct;
                    if (wprev <= kPcgBS) {
                        if (crc.s0 >= 0) t = dadd(t, prev[crc.s0]);
                        if (crc.s1 >= 0) t = dadd(t, prev[crc.s1]);
                        if (crc.s2 >= 0) t = dadd(t, prev[crc.s2]);
                    } else {
                        const int* nb = a.nbr + (size_t)(lsA + tid) * 6;
                        int mm;
                        if ((mm = nb[NB_MX]) >= 0) t = dadd(t, a.pq[mm]);
                        if ((mm = nb[NB_MY]) >= 0) t = dadd(t, a.pq[mm]);
                        if ((mm = nb[NB_MZ]) >= 0) t = dadd(t, a.pq[mm]);
                    }
                    double qv = dmul(t, crc.pc);
                    double pqv = dmul(crc.pc, qv);
                    cur[tid] = pqv;
                    a.q[lsA + tid] = qv;
                }
            } else {
                for (int ps = lsA + tid; ps < lsB; ps += sw) {
                    const int* nb = a.nbr + (size_t)ps * 6;
                    double t = r[ps];
                    int mm;
                    if (wprev <= kPcgBS) {
                        if ((mm = nb[NB_MX]) >= 0) t = dadd(t, prev[mm - lsP]);
                        if ((mm = nb[NB_MY]) >= 0) t = dadd(t, prev[mm - lsP]);
                        if ((mm = nb[NB_MZ]) >= 0) t = dadd(t, prev[mm - lsP]);
                    } else {
                        if ((mm = nb[NB_MX]) >= 0) t = dadd(t, a.pq[mm]);
                        if ((mm = nb[NB_MY]) >= 0) t = dadd(t, a.pq[mm]);
                        if ((mm = nb[NB_MZ]) >= 0) t = dadd(t, a.pq[mm]);
                    }
                    double pc = a.precon[ps];
                    double qv = dmul(t, pc);
                    double pqv = dmul(pc, qv);
                    a.q[ps] = qv;
                    a.pq[ps] = pqv;
                    if (wcur <= kPcgBS) cur[ps - lsA] = pqv;  // the next level reads the window
                }
            }
        }
        unsigned long long c1 = lt ? clock64() : 0;
        sweep_bar(nbar);
        if (lt) {
            unsigned long long c2 = clock64();
            lt[1] += c1 - c0;
            lt[2] += c2 - c1;
            lt[3] += 1;
        }
        if (wcur <= kPcgBS) {
            double* tt = prev;
            prev = cur;
            cur = tt;
        }
        ct = nt_;
        crc = nrc;
        lsP = lsA;
        lsA = lsB;
        lsB = lsC;
    }
    if (producer) asm volatile("cp.async.wait_all;" ::: "memory");
    sweep_bar(nbar);
    // ---------------- backward
    if (producer) {
        for (int d = 0; d < kStages - 1; ++d) produce_level(m, l1 - 1 - d, l0, l1, a.q, r, a.brec, lane);
        cp_wait_ahead();
    }
    sweep_bar(nbar);
    double* next = m.w0;
    cur = m.w1;
    int lsN = m.lvs[l1], lsH = m.lvs[min(l1 + 1, a.nlevels)];  // starts of levels L+1, L+2
    lsA = m.lvs[l1 - 1];
    double cq = 0.0, cr = 0.0;
    crc = SweepRec{};
    if (!producer && tid < lsN - lsA && lsN - lsA <= kSweepMax) {
        int slot = ((l1 - 1) % kStages) * kPcgBS + tid;
        cq = m.sa[slot];
        cr = m.sb[slot];
        crc = m.sr[slot];
    }
    for (int L = l1 - 1; L >= l0; --L) {
        int lsQ = L > 0 ? m.lvs[L - 1] : 0;
        const int wnext = lsH - lsN, wcur = lsN - lsA, wlow = lsA - lsQ;
        double nq = 0.0, nr = 0.0;
        SweepRec nrc{};
        if (producer) {
            produce_level(m, L - (kStages - 1), l0, l1, a.q, r, a.brec, lane);
            cp_wait_ahead();
        } else {
            if (L - 1 >= l0 && tid < wlow && wlow <= kSweepMax) {  // prefetch level L-1
                int slot = ((L - 1) % kStages) * kPcgBS + tid;
                nq = m.sa[slot];
                nr = m.sb[slot];
                nrc = m.sr[slot];
            }
            if (wcur <= kSweepMax) {
                if (tid < wcur) {
                    double t = cq, pc = crc.pc;
                    if (L + 1 < l1 && wnext <= kPcgBS) {
                        if (crc.s0 >= 0) t = dadd(t, dmul(pc, next[crc.s0]));
                        if (crc.s1 >= 0) t = dadd(t, dmul(pc, next[crc.s1]));
                        if (crc.s2 >= 0) t = dadd(t, dmul(pc, next[crc.s2]));
                    } else {
                        const int* nb = a.nbr + (size_t)(lsA + tid) * 6;
                        int mm;
                        if ((mm = nb[NB_PX]) >= 0) t = dadd(t, dmul(pc, z[mm]));
                        if ((mm = nb[NB_PY]) >= 0) t = dadd(t, dmul(pc, z[mm]));
                        if ((mm = nb[NB_PZ]) >= 0) t = dadd(t, dmul(pc, z[mm]));
                    }
                    double zv = dmul(t, pc);
                    cur[tid] = zv;
                    z[lsA + tid] = zv;
                    a.prod[a.exact_dots ? a.cinv[lsA + tid] : lsA + tid] = dmul(zv, cr);
                }
            } else {
                for (int ps = lsA + tid; ps < lsN; ps += sw) {
                    const int* nb = a.nbr + (size_t)ps * 6;
                    double pc = a.precon[ps];
                    double t = a.q[ps];
                    int mm;
                    if (L + 1 < l1 && wnext <= kPcgBS) {
                        if ((mm = nb[NB_PX]) >= 0) t = dadd(t, dmul(pc, next[mm - lsN]));
                        if ((mm = nb[NB_PY]) >= 0) t = dadd(t, dmul(pc, next[mm - lsN]));
                        if ((mm = nb[NB_PZ]) >= 0) t = dadd(t, dmul(pc, next[mm - lsN]));
                    } else {
                        if ((mm = nb[NB_PX]) >= 0) t = dadd(t, dmul(pc, z[mm]));
                        if ((mm = nb[NB_PY]) >= 0) t = dadd(t, dmul(pc, z[mm]));
                        if ((mm = nb[NB_PZ]) >= 0) t = dadd(t, dmul(pc, z[mm]));
                    }
                    double zv = dmul(t, pc);
                    z[ps] = zv;
                    if (wcur <= kPcgBS) cur[ps - lsA] = zv;  // the next level reads the window
                    a.prod[a.exact_dots ? a.cinv[ps] : ps] = dmul(zv, r[ps]);
                }
            }
        }
        sweep_bar(nbar);
        if (wcur <= kPcgBS) {
            double* tt = next;
            next = cur;
            cur = tt;
        }
        cq = nq;
        cr = nr;
        crc = nrc;
        lsH = lsN;
        lsN = lsA;
        lsA = lsQ;
    }
    if (producer) asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
}

// pcg (pressure.rs:341-397) as one thread-block cluster of C CTAs (C = 1
// when the GPU is shared with other scenes). CTA 0 runs the MIC(0) factor
// and both triangular sweeps in its shared memory exactly as a single block
// would (their cost is the per-level latency, which more SMs do not lower);
// the matvec, the updates of p, r and s, the norms and the dots are spread
// over all CTAs, whose extra bandwidth they are bound by. Phases are ordered
// by cluster barriers.
__device__ __forceinline__ void k_pcg_body(VB vb_, PcgArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double sh[40];
    PcgSmem m;
    {
        unsigned char* q = smem_raw;
        m.sr = (SweepRec*)q; q += (size_t)kStages * kPcgBS * 16;
        m.sa = (double*)q; q += (size_t)kStages * kPcgBS * 8;
        m.sb = (double*)q; q += (size_t)kStages * kPcgBS * 8;
        m.w0 = (double*)q; q += (size_t)kPcgBS * 8;
        m.w1 = (double*)q; q += (size_t)kPcgBS * 8;
        m.m0 = (int*)q; q += (size_t)kPcgBS * 4;
        m.m1 = (int*)q; q += (size_t)kPcgBS * 4;
        m.lvs = (int*)q;
    }
    PcgCl c = pcg_cl();
    const bool lead = c.rank == 0;  // the CTA that runs the sweeps
    if (a.nlevels > kMaxLevelsSmem) m.lvs = const_cast<int*>(a.level_start);
    else
        for (int L = threadIdx.x; L <= a.nlevels; L += blockDim.x) m.lvs[L] = a.level_start[L];
    __syncthreads();
    const uint32_t nf = *a.nf;
    const uint32_t ntile = (nf + kTile - 1) / kTile;
    const int tid = threadIdx.x, lane = tid & 31;
    // Non-empty level range and the widest level -> sweep width (warps).
    __shared__ int s_l0, s_l1, s_wmax;
    if (tid == 0) {
        s_l0 = a.nlevels;
        s_l1 = 0;
        s_wmax = 0;
    }
    __syncthreads();
    for (int L = tid; L < a.nlevels; L += blockDim.x) {
        int w = m.lvs[L + 1] - m.lvs[L];
        if (w > 0) {
            atomicMin(&s_l0, L);
            atomicMax(&s_l1, L + 1);
            atomicMax(&s_wmax, w);
        }
    }
    __syncthreads();
    const int l0 = s_l0, l1 = s_l1;
    const int sw = min(kSweepMax, max(32, (s_wmax + 31) & ~31));

    // Section timers (CTA 0, thread 0; kept in shared memory to spare registers).
    __shared__ unsigned long long tsec[8], ltim[4], tck;
    const bool timed = a.timing != nullptr && lead;
    if (tid == 0) {
        for (int q = 0; q < 8; ++q) tsec[q] = 0;
        for (int q = 0; q < 4; ++q) ltim[q] = 0;
        tck = clock64();
    }
    unsigned long long* lt = (timed && tid == 0) ? ltim : nullptr;
#define SECTION(idx)                                   \
    do {                                               \
        if (timed && tid == 0) {                       \
            unsigned long long now_ = clock64();       \
            tsec[idx] += now_ - tck;                   \
            tck = now_;                                \
        }                                              \
    } while (0)
    double mx = 0.0;
    for (uint32_t i = c.gt; i < nf; i += c.G) mx = fmax(mx, fabs(a.b[i]));
    double residual = pcg_cl_max<kPcgBS>(c, a, mx, sh);
    int iters = 0;
    if (residual > a.tol) {
        SECTION(7);
        if (lead) {
            pcg_build_mic0(a, m, sw, l0, l1);
            pcg_build_records(a, m, nf);
        }
        SECTION(0);
        for (uint32_t i = c.gt; i < nf; i += c.G) {
            a.r[i] = a.b[i];
            a.p[i] = 0.0;
        }
        cluster_sync_all();  // r complete before the sweeps read it
        if (lead) pcg_apply_mic0(a, m, a.r, a.z, sw, l0, l1);
        SECTION(1);
        // dot(z, r); its barriers also publish z
        double sigma = a.exact_dots ? pcg_exact_dot(a, c, sh) : pcg_tree_dot_own(a, lead, nf);
        SECTION(4);
        for (uint32_t i = c.gt; i < nf; i += c.G) a.s[i] = __ldcg(a.z + i);
        cluster_sync_all();  // s complete before the matvec reads neighbours
        for (int it = 0; it < a.max_iters; ++it) {
            iters = it + 1;
            // apply_a (pressure.rs:400-439): diag*x, then +x,-x,+y,-y,+z,-z; and s*As.
            // Tiles of kTile cells per warp (the tree dot's tiles): lane l takes
            // cells l, l+32, ... of the tile.
            for (uint32_t t = (uint32_t)c.gw; t < ntile; t += (uint32_t)c.nw) {
                double acc = 0.0;
#pragma unroll 2
                for (int u = 0; u < kTile / 32; ++u) {
                    const uint32_t i = t * kTile + lane + 32u * u;
                    if (i >= nf) break;
                    const int2* nb2 = reinterpret_cast<const int2*>(a.nbr + (size_t)i * 6);
                    const int2 x0 = nb2[0], x1 = nb2[1], x2 = nb2[2];
                    const int nbv[6] = {x0.x, x0.y, x1.x, x1.y, x2.x, x2.y};
                    const double sv = __ldcg(a.s + i);
                    double nsv[6];
#pragma unroll
                    for (int d = 0; d < 6; ++d) nsv[d] = nbv[d] >= 0 ? __ldcg(a.s + nbv[d]) : 0.0;
                    double v = dmul((double)a.diag[i], sv);
                    if (nbv[NB_PX] >= 0) v = dsub(v, nsv[NB_PX]);
                    if (nbv[NB_MX] >= 0) v = dsub(v, nsv[NB_MX]);
                    if (nbv[NB_PY] >= 0) v = dsub(v, nsv[NB_PY]);
                    if (nbv[NB_MY] >= 0) v = dsub(v, nsv[NB_MY]);
                    if (nbv[NB_PZ] >= 0) v = dsub(v, nsv[NB_PZ]);
                    if (nbv[NB_MZ] >= 0) v = dsub(v, nsv[NB_MZ]);
                    a.as[i] = v;
                    if (a.exact_dots) a.prod[a.cinv[i]] = dmul(sv, v);
                    else acc = dadd(acc, dmul(sv, v));
                }
                if (!a.exact_dots) {
                    acc = warp_tree_sum(acc);
                    if (lane == 0) a.tpart[t] = acc;
                }
            }
            SECTION(3);
            double denom;  // dot(s, As)
            if (a.exact_dots) {
                denom = pcg_exact_dot(a, c, sh);
            } else {
                cluster_sync_all();
                denom = pcg_tile_total(a, ntile);
            }
            SECTION(4);
            if (fabs(denom) < 1e-30) break;
            double alpha = ddiv(sigma, denom);
            double mr = 0.0;
            for (uint32_t i = c.gt; i < nf; i += c.G) {
                a.p[i] = dadd(a.p[i], dmul(alpha, __ldcg(a.s + i)));
                double rv = dsub(a.r[i], dmul(alpha, __ldcg(a.as + i)));
                a.r[i] = rv;
                mr = fmax(mr, fabs(rv));
            }
            residual = pcg_cl_max<kPcgBS>(c, a, mr, sh);  // its barrier also publishes r
            SECTION(5);
            if (residual <= a.tol) break;
            if (lead) pcg_apply_mic0(a, m, a.r, a.z, sw, l0, l1, lt);
            SECTION(1);
            double sigma_new = a.exact_dots ? pcg_exact_dot(a, c, sh) : pcg_tree_dot_own(a, lead, nf);  // dot(z, r)
            SECTION(4);
            double beta = ddiv(sigma_new, sigma);
            for (uint32_t i = c.gt; i < nf; i += c.G) a.s[i] = dadd(__ldcg(a.z + i), dmul(beta, a.s[i]));
            cluster_sync_all();
            SECTION(6);
            sigma = sigma_new;
        }
        for (uint32_t i = c.gt; i < nf; i += c.G) a.p_dense[a.lv_cell[i]] = a.p[i];
    }
    SECTION(7);
#undef SECTION
    if (lead && tid == 0) {
        *a.out_iters = iters;
        *a.out_residual = residual;
        if (a.timing) {
            for (int q = 0; q < 8; ++q) a.timing[q] += tsec[q];
            for (int q = 0; q < 4; ++q) a.timing[8 + q] += ltim[q];
            a.timing[12] += (unsigned long long)sw;
            a.timing[13] += (unsigned long long)(l1 - l0);
            a.timing[14] += 1;
        }
    }
}
__global__ void __launch_bounds__(kPcgBS, 1) k_pcg(PcgArgs a) { k_pcg_body(VB{blockIdx.x, gridDim.x}, a); }

// apply_pressure_gradient (pressure.rs:285-332): one thread per node owning
// its u/v/w faces; f64 update rounded back to the f32 face.
__device__ __forceinline__ void k_gradient_body(VB vb_, Grid g, const uint8_t* __restrict__ cells, const double* __restrict__ p,
                           double coef, float* __restrict__ u, float* __restrict__ v,
                           float* __restrict__ w) {
    int i, j, k;
    if (!node_of(g, (size_t)vb_.bid * blockDim.x + threadIdx.x, i, j, k)) return;
    size_t c = ((size_t)k * g.ny + j) * g.nx + i;
    if (j < g.ny && k < g.nz && i >= 1 && i < g.nx) {
        uint8_t l = cells[c - 1], r = cells[c];
        if (l != SOLID && r != SOLID && (l == FLUID || r == FLUID)) {
            size_t f = ((size_t)k * g.ny + j) * (g.nx + 1) + i;
            u[f] = (float)dsub((double)u[f], dmul(coef, dsub(p[c], p[c - 1])));
        }
    }
    if (i < g.nx && k < g.nz && j >= 1 && j < g.ny) {
        uint8_t l = cells[c - g.nx], r = cells[c];
        if (l != SOLID && r != SOLID && (l == FLUID || r == FLUID)) {
            size_t f = ((size_t)k * (g.ny + 1) + j) * g.nx + i;
            v[f] = (float)dsub((double)v[f], dmul(coef, dsub(p[c], p[c - g.nx])));
        }
    }
    if (i < g.nx && j < g.ny && k >= 1 && k < g.nz) {
        size_t s = (size_t)g.nx * g.ny;
        uint8_t l = cells[c - s], r = cells[c];
        if (l != SOLID && r != SOLID && (l == FLUID || r == FLUID)) {
            w[c] = (float)dsub((double)w[c], dmul(coef, dsub(p[c], p[c - s])));
        }
    }
}
__global__ void k_gradient(Grid g, const uint8_t* __restrict__ cells, const double* __restrict__ p,
                           double coef, float* __restrict__ u, float* __restrict__ v,
                           float* __restrict__ w) { k_gradient_body(VB{blockIdx.x, gridDim.x}, g, cells, p, coef, u, v, w); }

}  // namespace sdr
