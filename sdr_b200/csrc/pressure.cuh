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

namespace sdr {

constexpr int kDotChunk = 4096;
constexpr int kPcgBS = 1024;
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
                         const int* __restrict__ pos_of_cell, int* __restrict__ corder,
                         int* __restrict__ chunk_start, int nchunks, const uint32_t* __restrict__ nf) {
    size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n && cells[c] == FLUID) corder[off[c]] = pos_of_cell[c];
    if (c < n && c % kDotChunk == 0) chunk_start[c / kDotChunk] = (int)off[c];
    if (c == 0) chunk_start[nchunks] = (int)*nf;
}

struct PcgArgs {
    const uint32_t* nf;  // device fluid count
    int nlevels;
    int nchunks;
    const int* level_start;
    const int* nbr;
    const uint8_t* diag;
    const uint8_t* nmask;
    const int* corder;
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
    double* partials;  // nchunks
    double tol;
    int max_iters;
    const uint32_t* lv_cell;
    double* p_dense;   // pre-zeroed; fluid cells written at exit
    int* out_iters;
    double* out_residual;
};

// Exact reference dot (pressure.rs:588-603): chunk partials in parallel, each
// a sequential sum over its fluid cells in cell order, then the partials in
// chunk order. Empty chunks contribute +0.0.
__device__ __forceinline__ double pcg_dot(const PcgArgs& a, const double* x, const double* y,
                                          double* sh) {
    for (int ch = threadIdx.x; ch < a.nchunks; ch += blockDim.x) {
        int e = a.chunk_start[ch + 1];
        double acc = 0.0;
        for (int t = a.chunk_start[ch]; t < e; ++t) {
            int ps = a.corder[t];
            acc = dadd(acc, dmul(x[ps], y[ps]));
        }
        a.partials[ch] = acc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = -0.0;
        for (int ch = 0; ch < a.nchunks; ++ch) s = dadd(s, a.partials[ch]);
        sh[0] = s;
    }
    __syncthreads();
    double r = sh[0];
    __syncthreads();
    return r;
}

// build_mic0 (pressure.rs:442-513) as a forward level sweep; precon values of
// level L-1 are read from the shared window (or global when the level is wider).
__device__ void pcg_build_mic0(const PcgArgs& a, double* win0, double* win1) {
    const double TAU = 0.97, SIGMA = 0.25;
    double* prev = win0;
    double* cur = win1;
    for (int L = 0; L < a.nlevels; ++L) {
        int ls = a.level_start[L], le = a.level_start[L + 1];
        int lsp = L > 0 ? a.level_start[L - 1] : 0;
        bool prev_in = L > 0 && (ls - lsp) <= kPcgWin;
        bool cur_in = (le - ls) <= kPcgWin;
        for (int ps = ls + threadIdx.x; ps < le; ps += blockDim.x) {
            const int* nb = a.nbr + (size_t)ps * 6;
            double axi = 0, pxi = 0, axi_y = 0, axi_z = 0;
            double ayj = 0, pyj = 0, ayj_x = 0, ayj_z = 0;
            double azk = 0, pzk = 0, azk_x = 0, azk_y = 0;
            int m = nb[NB_MX];
            if (m >= 0) {
                uint8_t mk = a.nmask[m];
                axi = -1.0;
                pxi = prev_in ? prev[m - lsp] : a.precon[m];
                axi_y = (mk >> NB_PY & 1) ? -1.0 : 0.0;
                axi_z = (mk >> NB_PZ & 1) ? -1.0 : 0.0;
            }
            m = nb[NB_MY];
            if (m >= 0) {
                uint8_t mk = a.nmask[m];
                ayj = -1.0;
                pyj = prev_in ? prev[m - lsp] : a.precon[m];
                ayj_x = (mk >> NB_PX & 1) ? -1.0 : 0.0;
                ayj_z = (mk >> NB_PZ & 1) ? -1.0 : 0.0;
            }
            m = nb[NB_MZ];
            if (m >= 0) {
                uint8_t mk = a.nmask[m];
                azk = -1.0;
                pzk = prev_in ? prev[m - lsp] : a.precon[m];
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
            if (cur_in) cur[ps - ls] = pc;
        }
        __syncthreads();
        double* t = prev;
        prev = cur;
        cur = t;
    }
}

// apply_mic0 (pressure.rs:517-570): forward L q = r then backward L^T z = q.
// Forward:  t = r + pq[-x] + pq[-y] + pq[-z]  (pq = precon*q of the predecessor,
//           which is what `t -= plus*precon*q` with plus = -1 adds), q = t*pc.
// Backward: t = q + pc*z[+x] + pc*z[+y] + pc*z[+z], z = t*pc.
__device__ void pcg_apply_mic0(const PcgArgs& a, const double* r, double* z, double* win0,
                               double* win1) {
    double* prev = win0;
    double* cur = win1;
    for (int L = 0; L < a.nlevels; ++L) {
        int ls = a.level_start[L], le = a.level_start[L + 1];
        int lsp = L > 0 ? a.level_start[L - 1] : 0;
        bool prev_in = L > 0 && (ls - lsp) <= kPcgWin;
        bool cur_in = (le - ls) <= kPcgWin;
        for (int ps = ls + threadIdx.x; ps < le; ps += blockDim.x) {
            const int* nb = a.nbr + (size_t)ps * 6;
            double t = r[ps];
            int m = nb[NB_MX];
            if (m >= 0) t = dadd(t, prev_in ? prev[m - lsp] : a.pq[m]);
            m = nb[NB_MY];
            if (m >= 0) t = dadd(t, prev_in ? prev[m - lsp] : a.pq[m]);
            m = nb[NB_MZ];
            if (m >= 0) t = dadd(t, prev_in ? prev[m - lsp] : a.pq[m]);
            double pc = a.precon[ps];
            double qv = dmul(t, pc);
            double pqv = dmul(pc, qv);
            a.q[ps] = qv;
            a.pq[ps] = pqv;
            if (cur_in) cur[ps - ls] = pqv;
        }
        __syncthreads();
        double* t = prev;
        prev = cur;
        cur = t;
    }
    double* next = win0;
    cur = win1;
    for (int L = a.nlevels - 1; L >= 0; --L) {
        int ls = a.level_start[L], le = a.level_start[L + 1];
        int lsn = a.level_start[L + 1];
        int len_next = L + 1 < a.nlevels ? a.level_start[L + 2] - lsn : 0;
        bool next_in = L + 1 < a.nlevels && len_next <= kPcgWin;
        bool cur_in = (le - ls) <= kPcgWin;
        for (int ps = ls + threadIdx.x; ps < le; ps += blockDim.x) {
            const int* nb = a.nbr + (size_t)ps * 6;
            double pc = a.precon[ps];
            double t = a.q[ps];
            int m = nb[NB_PX];
            if (m >= 0) t = dadd(t, dmul(pc, next_in ? next[m - lsn] : z[m]));
            m = nb[NB_PY];
            if (m >= 0) t = dadd(t, dmul(pc, next_in ? next[m - lsn] : z[m]));
            m = nb[NB_PZ];
            if (m >= 0) t = dadd(t, dmul(pc, next_in ? next[m - lsn] : z[m]));
            double zv = dmul(t, pc);
            z[ps] = zv;
            if (cur_in) cur[ps - ls] = zv;
        }
        __syncthreads();
        double* t = next;
        next = cur;
        cur = t;
    }
}

// pcg (pressure.rs:341-397) in one persistent block.
__global__ void __launch_bounds__(kPcgBS, 1) k_pcg(PcgArgs a) {
    extern __shared__ double win[];
    __shared__ double sh[40];
    double* win0 = win;
    double* win1 = win + kPcgWin;
    const uint32_t nf = *a.nf;
    const int tid = threadIdx.x, nt = blockDim.x;

    double m = 0.0;
    for (uint32_t i = tid; i < nf; i += nt) m = fmax(m, fabs(a.b[i]));
    double residual = block_max<kPcgBS>(m, sh);
    int iters = 0;
    if (residual > a.tol) {
        pcg_build_mic0(a, win0, win1);
        for (uint32_t i = tid; i < nf; i += nt) {
            a.r[i] = a.b[i];
            a.p[i] = 0.0;
        }
        __syncthreads();
        pcg_apply_mic0(a, a.r, a.z, win0, win1);
        for (uint32_t i = tid; i < nf; i += nt) a.s[i] = a.z[i];
        __syncthreads();
        double sigma = pcg_dot(a, a.z, a.r, sh);
        for (int it = 0; it < a.max_iters; ++it) {
            iters = it + 1;
            // apply_a (pressure.rs:400-439): diag*x, then +x,-x,+y,-y,+z,-z
            for (uint32_t i = tid; i < nf; i += nt) {
                const int* nb = a.nbr + (size_t)i * 6;
                double v = dmul((double)a.diag[i], a.s[i]);
                int o;
                if ((o = nb[NB_PX]) >= 0) v = dsub(v, a.s[o]);
                if ((o = nb[NB_MX]) >= 0) v = dsub(v, a.s[o]);
                if ((o = nb[NB_PY]) >= 0) v = dsub(v, a.s[o]);
                if ((o = nb[NB_MY]) >= 0) v = dsub(v, a.s[o]);
                if ((o = nb[NB_PZ]) >= 0) v = dsub(v, a.s[o]);
                if ((o = nb[NB_MZ]) >= 0) v = dsub(v, a.s[o]);
                a.as[i] = v;
            }
            __syncthreads();
            double denom = pcg_dot(a, a.s, a.as, sh);
            if (fabs(denom) < 1e-30) break;
            double alpha = ddiv(sigma, denom);
            double mr = 0.0;
            for (uint32_t i = tid; i < nf; i += nt) {
                a.p[i] = dadd(a.p[i], dmul(alpha, a.s[i]));
                double rv = dsub(a.r[i], dmul(alpha, a.as[i]));
                a.r[i] = rv;
                mr = fmax(mr, fabs(rv));
            }
            residual = block_max<kPcgBS>(mr, sh);
            if (residual <= a.tol) break;
            pcg_apply_mic0(a, a.r, a.z, win0, win1);
            double sigma_new = pcg_dot(a, a.z, a.r, sh);
            double beta = ddiv(sigma_new, sigma);
            for (uint32_t i = tid; i < nf; i += nt) a.s[i] = dadd(a.z[i], dmul(beta, a.s[i]));
            __syncthreads();
            sigma = sigma_new;
        }
        for (uint32_t i = tid; i < nf; i += nt) a.p_dense[a.lv_cell[i]] = a.p[i];
    }
    if (tid == 0) {
        *a.out_iters = iters;
        *a.out_residual = residual;
    }
}

// apply_pressure_gradient (pressure.rs:285-332): one thread per node owning
// its u/v/w faces; f64 update rounded back to the f32 face.
__global__ void k_gradient(Grid g, const uint8_t* __restrict__ cells, const double* __restrict__ p,
                           double coef, float* __restrict__ u, float* __restrict__ v,
                           float* __restrict__ w) {
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i > g.nx) return;
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
