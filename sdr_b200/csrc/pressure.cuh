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
__global__ void k_lines_count(Grid g, const uint8_t* __restrict__ cells, int nlevels,
                              uint32_t* __restrict__ cnt) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
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

// Assign wavefront positions: pos = line base + rank along j.
__global__ void k_lines_assign(Grid g, const uint8_t* __restrict__ cells, int nlevels,
                               const uint32_t* __restrict__ base, int* __restrict__ pos_of_cell,
                               uint32_t* __restrict__ lv_cell) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
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

// Level starts from the (level, k) line bases; nf is the device fluid count.
__global__ void k_level_starts_dev(const uint32_t* __restrict__ base, int nlevels, int nz,
                                   const uint32_t* __restrict__ nf, int* __restrict__ level_start) {
    int L = blockIdx.x * blockDim.x + threadIdx.x;
    if (L < nlevels) level_start[L] = (int)base[L * nz];
    if (L == nlevels) level_start[L] = (int)*nf;
}

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
__global__ void k_tables(TableArgs a) {
    uint32_t pos = blockIdx.x * blockDim.x + threadIdx.x;
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

// Fluid cells in cell-index order -> wavefront position, for the chunked dot.
__global__ void k_fluid_flags(const uint8_t* __restrict__ cells, size_t n, uint32_t* __restrict__ flag) {
    size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n) flag[c] = cells[c] == FLUID;
}

__global__ void k_corder(const uint8_t* __restrict__ cells, size_t n, const uint32_t* __restrict__ off,
                         const int* __restrict__ pos_of_cell, int* __restrict__ corder, int* __restrict__ cinv,
                         int* __restrict__ chunk_start, int nchunks, const uint32_t* __restrict__ nf) {
    size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n && cells[c] == FLUID) {
        corder[off[c]] = pos_of_cell[c];
        cinv[pos_of_cell[c]] = (int)off[c];
    }
    if (c < n && c % kDotChunk == 0) chunk_start[c / kDotChunk] = (int)off[c];
    if (c == 0) chunk_start[nchunks] = (int)*nf;
}

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
    double* prod;       // per-cell products in cell order (reference dot order)
    double* partials;   // nchunks (global fallback when they do not fit in shared memory)
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
// neighbour masks, the level starts and the dot partials.
constexpr int kStages = 4;          // levels in flight ahead of the sweep
constexpr int kMaxLevelsSmem = 2048;
constexpr int kMaxChunksSmem = 2048;
constexpr int kSweepMax = kPcgBS - 32;  // compute threads; one producer warp stages ahead
constexpr size_t kPcgSmem = (size_t)kStages * kPcgBS * (8 + 8 + 16) + 2 * kPcgBS * 8 + 2 * kPcgBS * 4 +
                            (kMaxLevelsSmem + 1) * 4 + kMaxChunksSmem * 8;

struct PcgSmem {
    double* sa;     // [kStages][BS]
    double* sb;     // [kStages][BS]
    SweepRec* sr;   // [kStages][BS]
    double* w0;     // [BS] level window
    double* w1;
    int* m0;        // [BS] neighbour-mask window (MIC build)
    int* m1;
    int* lvs;       // level starts (smem copy or global)
    double* part;   // dot partials
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

// Exact reference dot (pressure.rs:588-603) over `prod` (cell order): one
// warp per 4096-cell chunk folds its products in cell order from registers
// through shuffles, then one thread sums the partials in chunk order.
__device__ __forceinline__ double pcg_chunk_sums(const PcgArgs& a, const PcgSmem& m, double* sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int ch = warp; ch < a.nchunks; ch += nw) {
        int t = a.chunk_start[ch], e = a.chunk_start[ch + 1];
        double acc = 0.0;
        for (; t < e; t += 512) {
            double v[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) {
                int idx = t + u * 32 + lane;
                v[u] = idx < e ? a.prod[idx] : 0.0;
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
        if (lane == 0) m.part[ch] = acc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = -0.0;
        for (int ch = 0; ch < a.nchunks; ++ch) s = dadd(s, m.part[ch]);
        sh[0] = s;
    }
    __syncthreads();
    double r = sh[0];
    __syncthreads();
    return r;
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
__device__ double pcg_apply_mic0(const PcgArgs& a, const PcgSmem& m, const double* r, double* z, int sw, int l0,
                                 int l1, unsigned long long* lt = nullptr) {
    const int tid = threadIdx.x;
    const int nbar = sw + 32;
    double zr = 0.0;
    if (tid >= nbar) {
        __syncthreads();
        return zr;
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
                    double pr = dmul(zv, cr);
                    if (a.exact_dots) a.prod[a.cinv[lsA + tid]] = pr;
                    else zr = dadd(zr, pr);
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
                    double pr = dmul(zv, r[ps]);
                    if (a.exact_dots) a.prod[a.cinv[ps]] = pr;
                    else zr = dadd(zr, pr);
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
    return zr;
}

// pcg (pressure.rs:341-397) in one persistent block.
__global__ void __launch_bounds__(kPcgBS, 1) k_pcg(PcgArgs a) {
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
        m.part = (double*)q; q += (size_t)kMaxChunksSmem * 8;
        m.m0 = (int*)q; q += (size_t)kPcgBS * 4;
        m.m1 = (int*)q; q += (size_t)kPcgBS * 4;
        m.lvs = (int*)q;
    }
    if (a.nlevels > kMaxLevelsSmem) m.lvs = const_cast<int*>(a.level_start);
    else
        for (int L = threadIdx.x; L <= a.nlevels; L += blockDim.x) m.lvs[L] = a.level_start[L];
    if (a.nchunks > kMaxChunksSmem) m.part = a.partials;
    __syncthreads();
    const uint32_t nf = *a.nf;
    const int tid = threadIdx.x, nt = blockDim.x;
    // Non-empty level range and the widest level -> sweep width (warps).
    __shared__ int s_l0, s_l1, s_wmax;
    if (tid == 0) {
        s_l0 = a.nlevels;
        s_l1 = 0;
        s_wmax = 0;
    }
    __syncthreads();
    for (int L = tid; L < a.nlevels; L += nt) {
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

    // Section timers (thread 0 only, kept in shared memory to spare registers).
    __shared__ unsigned long long tsec[8], ltim[4], tck;
    const bool timed = a.timing != nullptr;
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
    for (uint32_t i = tid; i < nf; i += nt) mx = fmax(mx, fabs(a.b[i]));
    double residual = block_max<kPcgBS>(mx, sh);
    int iters = 0;
    if (residual > a.tol) {
        SECTION(7);
        pcg_build_mic0(a, m, sw, l0, l1);
        pcg_build_records(a, m, nf);
        SECTION(0);
        for (uint32_t i = tid; i < nf; i += nt) {
            a.r[i] = a.b[i];
            a.p[i] = 0.0;
        }
        __syncthreads();
        double zr = pcg_apply_mic0(a, m, a.r, a.z, sw, l0, l1);
        SECTION(1);
        for (uint32_t i = tid; i < nf; i += nt) a.s[i] = a.z[i];
        __syncthreads();
        double sigma = a.exact_dots ? pcg_chunk_sums(a, m, sh) : block_sum<kPcgBS>(zr, sh);  // dot(z, r)
        SECTION(4);
        for (int it = 0; it < a.max_iters; ++it) {
            iters = it + 1;
            // apply_a (pressure.rs:400-439): diag*x, then +x,-x,+y,-y,+z,-z; and s*As.
            // Two cells per thread per round, index loads first for memory parallelism.
            double sas = 0.0;
            for (uint32_t i0 = tid; i0 < nf; i0 += 2 * nt) {
                int nbv[2][6];
                double sv[2];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    uint32_t i = i0 + u * nt;
                    if (i < nf) {
                        const int2* nb2 = reinterpret_cast<const int2*>(a.nbr + (size_t)i * 6);
                        int2 x0 = nb2[0], x1 = nb2[1], x2 = nb2[2];
                        nbv[u][0] = x0.x; nbv[u][1] = x0.y; nbv[u][2] = x1.x;
                        nbv[u][3] = x1.y; nbv[u][4] = x2.x; nbv[u][5] = x2.y;
                        sv[u] = a.s[i];
                    }
                }
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    uint32_t i = i0 + u * nt;
                    if (i < nf) {
                        double nsv[6];
#pragma unroll
                        for (int d = 0; d < 6; ++d) nsv[d] = nbv[u][d] >= 0 ? a.s[nbv[u][d]] : 0.0;
                        double v = dmul((double)a.diag[i], sv[u]);
                        if (nbv[u][NB_PX] >= 0) v = dsub(v, nsv[NB_PX]);
                        if (nbv[u][NB_MX] >= 0) v = dsub(v, nsv[NB_MX]);
                        if (nbv[u][NB_PY] >= 0) v = dsub(v, nsv[NB_PY]);
                        if (nbv[u][NB_MY] >= 0) v = dsub(v, nsv[NB_MY]);
                        if (nbv[u][NB_PZ] >= 0) v = dsub(v, nsv[NB_PZ]);
                        if (nbv[u][NB_MZ] >= 0) v = dsub(v, nsv[NB_MZ]);
                        a.as[i] = v;
                        if (a.exact_dots) a.prod[a.cinv[i]] = dmul(sv[u], v);
                        else sas = dadd(sas, dmul(sv[u], v));
                    }
                }
            }
            __syncthreads();
            SECTION(3);
            double denom = a.exact_dots ? pcg_chunk_sums(a, m, sh) : block_sum<kPcgBS>(sas, sh);  // dot(s, As)
            SECTION(4);
            if (fabs(denom) < 1e-30) break;
            double alpha = ddiv(sigma, denom);
            double mr = 0.0;
#pragma unroll 4
            for (uint32_t i = tid; i < nf; i += nt) {
                a.p[i] = dadd(a.p[i], dmul(alpha, a.s[i]));
                double rv = dsub(a.r[i], dmul(alpha, a.as[i]));
                a.r[i] = rv;
                mr = fmax(mr, fabs(rv));
            }
            residual = block_max<kPcgBS>(mr, sh);
            SECTION(5);
            if (residual <= a.tol) break;
            zr = pcg_apply_mic0(a, m, a.r, a.z, sw, l0, l1, lt);
            SECTION(1);
            double sigma_new = a.exact_dots ? pcg_chunk_sums(a, m, sh) : block_sum<kPcgBS>(zr, sh);  // dot(z, r)
            SECTION(4);
            double beta = ddiv(sigma_new, sigma);
#pragma unroll 4
            for (uint32_t i = tid; i < nf; i += nt) a.s[i] = dadd(a.z[i], dmul(beta, a.s[i]));
            __syncthreads();
            SECTION(6);
            sigma = sigma_new;
        }
        for (uint32_t i = tid; i < nf; i += nt) a.p_dense[a.lv_cell[i]] = a.p[i];
    }
    SECTION(7);
#undef SECTION
    if (tid == 0) {
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

// apply_pressure_gradient (pressure.rs:285-332): one thread per node owning
// its u/v/w faces; f64 update rounded back to the f32 face.
__global__ void k_gradient(Grid g, const uint8_t* __restrict__ cells, const double* __restrict__ p,
                           double coef, float* __restrict__ u, float* __restrict__ v,
                           float* __restrict__ w) {
    int i, j, k;
    if (!node_of(g, (size_t)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) return;
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

}  // namespace sdr
