// pcg (src/pressure.rs:341-397) over the whole GPU, for large fluid regions.
//
// The MIC(0) factor (pressure.rs:442-513) and its two triangular sweeps
// (pressure.rs:517-570) are recurrences along i+j+k. Here the grid's (j, k)
// lines are cut into tiles of kTwJ x kTwK lines, one CTA per tile and one
// thread per line. A tile walks the levels L = i+j+k of its cells in order;
// within a level every line has at most one cell (i = L - j - k), whose -x
// predecessor is the thread's own previous cell (a register) and whose -y and
// -z predecessors are the neighbouring lines' cells of level L-1 (shared
// memory, double-buffered by level), or, on the tile's low faces, cells of
// the neighbouring tiles. So a level costs one barrier of the tile's threads,
// and tiles synchronise only with their two upstream neighbours through
// exchange entries that mark their own readiness: a tile runs as soon as its
// neighbours are one level ahead, and a sweep takes about (levels x the level step) + (tile hops
// x the hand-off latency) instead of one grid-wide barrier per level. The
// backward sweep mirrors it (tiles wait on their +y / +z neighbours, levels in
// decreasing order).
//
// Per cell the arithmetic is that of k_pcg / k_pcg_cluster (the same operands
// in the same order), so the factor and both sweeps give the same bits, and so
// does the solve: the matvec, the updates and the dots run in the wavefront
// order and tiling of the other kernels, spread over the grid. The sweeps'
// operands live in rows: per tile one row of kTwLines entries per level of its
// range, so the lines of a level are contiguous and every copy and store of a
// level is coalesced (the lines' cells lie some 70 cells apart in cell order,
// which made each warp access touch 32 cache lines). The update phase writes
// the residual into the rows and the dots read z back through the wavefront
// index -> row map. Each compute thread keeps its next kTwDepth levels'
// operands in flight to shared memory (cp.async), so a level's step never
// waits on a global load.
//
// Synchronisation: one cooperative launch (every CTA resident). Phases are
// separated by a grid barrier (an arrival counter and a generation word,
// release/acquire at GPU scope). In a sweep the 8 compute warps of a CTA share
// a named barrier per level; a ninth warp polls the upstream tiles' exchange
// entries and copies their boundary values into a shared-memory ring, so
// compute threads never wait on a global load. Every wait gives up after about a
// second (2^31 SM cycles) or as soon as another CTA has given up, sets an
// error bit and lets the kernel wind down.
#pragma once
#include "pressure.cuh"

namespace sdr {

constexpr int kTwJ = 16;                     // lines per tile along y
constexpr int kTwK = 16;                     // lines per tile along z
constexpr int kTwLines = kTwJ * kTwK;        // compute threads: one per line
constexpr int kTwBS = kTwLines + 32;         // plus the progress warp
constexpr int kTwWarps = kTwBS / 32;
constexpr int kTwRing = 32;                  // levels of neighbour boundary values staged ahead
constexpr int kTwDepth = 6;                  // cells of each line whose operands are in flight to shared memory
constexpr long long kTwWaitCycles = 1ll << 31;  // ~1.1 s at 1965 MHz
constexpr uint32_t kTwErrWait = 16u;         // error bit: a sweep or barrier wait gave up
constexpr uint32_t kTwNoCell = 0xFFFFFFFFu;  // a row entry without a fluid cell
constexpr int kTwFace = 16;                  // lines of a tile face (either face)
// Levels a progress-warp poll loads at once: more loads in flight per poll
// slow the compute warps' shared-memory accesses on the same SM (pool solve
// at 0.2 mm: 76.3 ms with 2, 77.1 with 4, 79.7 with 8).
constexpr int kTwPoll = 2;
static_assert(kTwJ == kTwFace && kTwK == kTwFace, "both tile faces hold kTwFace lines");

struct TwArgs {
    PcgArgs a;                   // wavefront-order vectors, tables and dots (as k_pcg)
    int nx, ny, nz;
    int tj, tk, ntiles;          // tiles along y and z
    const uint32_t* coff;        // dense cell -> cell-order index of its fluid cell (exclusive scan, ncell + 1)
    uint32_t* icm_c;             // cell order: i | fluid-neighbour bits (NB_*) << 16 | non-solid count << 24
    // The sweeps' operands in rows: per tile, one row of kTwLines entries per
    // level of its range (entry = rbase[tile] + (L - tlo[tile]) * kTwLines +
    // line), so the lines of a level are contiguous and every access of a
    // level is coalesced. Entries without a fluid cell hold kTwNoCell in icm.
    uint32_t* icm;               // rows: the (i, mask, count) word, or kTwNoCell
    double2* rp;                 // rows: (residual, MIC(0) factor), the forward sweep's operands
    double2* qp;                 // rows: (forward sweep result, MIC(0) factor), the backward sweep's
    double* zr;                  // rows: backward sweep result
    uint32_t* tpos;              // wavefront index -> row entry of its cell
    uint32_t* rbase;             // per tile: its first row entry (ntiles + 1 entries)
    size_t rows_cap;             // row entries allocated
    // Exchange planes, level-major like the rows: a tile's boundary values of
    // its q-th level (sweep order) at rbase[tile] / kTwFace + q * kTwFace + l,
    // l the line along the face; the z face plane follows the y face plane
    // (rows_cap / kTwFace entries each). A level's values are one 128-byte line.
    double* exf;                 // forward sweeps: the +y face, then the +z face
    double* exb;                 // backward sweeps: the -y face, then the -z face
    int* tlo;                    // per tile: first and last level of its fluid cells
    int* thi;
    unsigned* bar;               // grid barrier: [0] arrivals, [1] generation
    double* gslots;              // 2 x gridDim CTA partials of grid maxima
    uint32_t* err;               // error bits
};

// ---------------------------------------------------------------- memory-order helpers
__device__ __forceinline__ unsigned long long ld_acquire_cta_sh(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.cta.shared::cta.u64 %0, [%1];" : "=l"(v) : "r"(smem_addr(p)) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_cta_sh(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.cta.shared::cta.u64 [%0], %1;" ::"r"(smem_addr(p)), "l"(v) : "memory");
}
// Exchange-plane entries: written and polled with relaxed GPU-scope accesses.
// kTwEmpty is a signalling-NaN pattern no arithmetic produces (IEEE results
// are quiet NaNs), so it can mark an entry not yet written.
constexpr unsigned long long kTwEmpty = 0x7FF4DEADBEEF0001ull;
__device__ __forceinline__ double ld_relaxed_gpu_f64(const double* p) {
    double v;
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_gpu_f64(double* p, double v) {
    asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed_gpu_u64(double* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
// 4-byte asynchronous copy into shared memory (cp_async16 and cp_commit are
// pressure.cuh's), and a wait until at most N of this thread's groups are pending.
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
template <int N>
__device__ __forceinline__ void cp_wait_n() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
__device__ __forceinline__ bool tw_failed(const TwArgs& t) { return *(volatile uint32_t*)t.err != 0u; }
// Barrier of the compute warps (named barrier 1).
__device__ __forceinline__ void tw_bar() { asm volatile("bar.sync 1, %0;" ::"n"(kTwLines) : "memory"); }

struct TwShared {
    double v[2][kTwLines];            // this tile's values of the last two levels, by line
    uint8_t m[2][kTwLines];           // the factorisation's neighbour masks, by line
    double ring[2][kTwRing][16];      // upstream neighbours' boundary values by level ([0] y face, [1] z face)
    uint8_t ringm[2][kTwRing][16];    // their masks (factorisation)
    double2 rec[kTwDepth][kTwLines];  // each line's next cells: (r or q, factor), by cell ordinal mod kTwDepth
    uint32_t icm[kTwDepth][kTwLines]; // and their (i, mask, count) words
    unsigned long long mine;          // levels this tile has completed (sweep order), for the progress warp
    unsigned long long avail[2];      // levels whose y / z neighbour values are in the ring
    int ok;
    double red[kTwWarps];
};

// Grid barrier; false if the wait gave up or another CTA has (the error bit is set).
__device__ bool tw_grid_sync(const TwArgs& t, TwShared& sh) {
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned gen = ld_acquire_gpu_u32(t.bar + 1);
        const unsigned arrived = atom_add_acqrel_gpu(t.bar, 1u) + 1u;
        if (arrived == gridDim.x) {
            t.bar[0] = 0u;  // ordered before the release of the next generation
            st_release_gpu_u32(t.bar + 1, gen + 1u);
        } else {
            const long long t0 = clock64();
            while (ld_acquire_gpu_u32(t.bar + 1) == gen) {
                if (tw_failed(t)) {
                    ok = 0;
                    break;
                }
                if (clock64() - t0 > kTwWaitCycles) {
                    atomicOr(t.err, kTwErrWait);
                    ok = 0;
                    break;
                }
            }
        }
        if (ok && tw_failed(t)) ok = 0;  // another CTA gave up: wind down
        sh.ok = ok;
    }
    __syncthreads();
    return sh.ok != 0;
}

__device__ __forceinline__ double tw_block_max(double v, TwShared& sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) sh.red[threadIdx.x >> 5] = v;
    __syncthreads();
    double m = sh.red[0];
    for (int w = 1; w < kTwWarps; ++w) m = fmax(m, sh.red[w]);
    __syncthreads();
    return m;
}

// Maximum over the grid (order-free): CTA maxima through a double-buffered slot array.
__device__ bool tw_grid_max(const TwArgs& t, TwShared& sh, double v, int& parity, double& out) {
    const double bm = tw_block_max(v, sh);
    double* sl = t.gslots + (size_t)parity * gridDim.x;
    parity ^= 1;
    if (threadIdx.x == 0) sl[blockIdx.x] = bm;
    if (!tw_grid_sync(t, sh)) return false;
    if (threadIdx.x < 32) {
        double m = 0.0;
        for (unsigned q = threadIdx.x; q < gridDim.x; q += 32) m = fmax(m, __ldcg(sl + q));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0) sh.red[0] = m;
    }
    __syncthreads();
    out = sh.red[0];
    __syncthreads();
    return true;
}

// Total of the tree-order tile sums (the lane pattern and xor tree of
// pcg_tile_total), formed by warp 0 and handed to the CTA.
__device__ double tw_tile_total(const TwArgs& t, uint32_t ntile, TwShared& sh) {
    if (threadIdx.x < 32) {
        const double s = pcg_tile_total(t.a, ntile);
        if (threadIdx.x == 0) sh.red[0] = s;
    }
    __syncthreads();
    const double r = sh.red[0];
    __syncthreads();
    return r;
}

// The reference's chunked dot (pressure.rs:588-603) over `prod` in cell
// order: one warp per 4096-cell chunk across the grid, then the chunk sums in
// chunk order (as pcg_exact_dot).
__device__ bool tw_exact_dot(const TwArgs& t, TwShared& sh, double& out) {
    const PcgArgs& a = t.a;
    if (!tw_grid_sync(t, sh)) return false;  // products complete
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * kTwWarps + (threadIdx.x >> 5), nw = gridDim.x * kTwWarps;
    for (int ch = gw; ch < a.nchunks; ch += nw) {
        int q = a.chunk_start[ch];
        const int e = a.chunk_start[ch + 1];
        double acc = 0.0;
        for (; q < e; q += 512) {
            double v[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) {
                const int idx = q + u * 32 + lane;
                v[u] = idx < e ? __ldcg(a.prod + idx) : 0.0;
            }
            const int cnt = min(512, e - q);
#pragma unroll
            for (int u = 0; u < 16; ++u) {
#pragma unroll 8
                for (int src = 0; src < 32; ++src) {
                    const double x = __shfl_sync(0xffffffffu, v[u], src);
                    if (u * 32 + src < cnt) acc = dadd(acc, x);
                }
            }
        }
        if (lane == 0) a.partials[ch] = acc;
    }
    if (!tw_grid_sync(t, sh)) return false;
    if (threadIdx.x == 0) {
        double s = -0.0;
        for (int ch = 0; ch < a.nchunks; ++ch) s = dadd(s, __ldcg(a.partials + ch));
        sh.red[0] = s;
    }
    __syncthreads();
    out = sh.red[0];
    __syncthreads();
    return true;
}

// ---------------------------------------------------------------- the tile sweeps
enum { TW_BUILD = 0, TW_FORWARD = 1, TW_BACKWARD = 2 };

// The progress warp of one tile's sweep: it stages the upstream tiles'
// boundary values into the shared ring, lanes 0-15 the y face (line
// (jb, k0 + l)), lanes 16-31 the z face (line (j0 + l, kb)), and publishes per
// face how many levels are staged. The values carry their own readiness: every
// entry of an exchange plane holds kTwEmpty until its producer writes it (the
// planes are filled when the solve lays out its rows), a lane polls the entries its
// next levels need (relaxed loads, kTwPoll levels at a time), and resets
// each entry it staged to kTwEmpty (the producer writes it again only in the
// next sweep of this direction, after a grid barrier). So a hand-off costs
// the producer's store reaching L2 and one poll, with no progress flags and no
// GPU-scope fences. A level needs no entry where the producer tile has no
// level before it (its range is in tlo/thi) or the cell lies outside the grid:
// the ring gets 0 there. The factorisation also stages the upstream cell's
// neighbour mask, read from the static cell tables.
template <int MODE>
__device__ void tw_progress_warp(const TwArgs& t, TwShared& sh, int tile, int nby, int nbz, int s_first,
                                 int s_last, int nlevels) {
    constexpr bool fwd = MODE != TW_BACKWARD;
    const int lane = threadIdx.x & 31;
    const int J = tile % t.tj, K = tile / t.tj;
    const int j0 = J * kTwJ, k0 = K * kTwK, nx = t.nx;
    const int face = lane >> 4, l = lane & 15;
    const int nb = face == 0 ? nby : nbz;
    // this tile's boundary line and the producer's line beside it
    const int jl = face == 0 ? (fwd ? j0 : j0 + kTwJ - 1) : j0 + l;
    const int kl = face == 0 ? k0 + l : (fwd ? k0 : k0 + kTwK - 1);
    const int jp = face == 0 ? (fwd ? jl - 1 : jl + 1) : jl;
    const int kp = face == 0 ? kl : (fwd ? kl - 1 : kl + 1);
    const bool line_ok = nb >= 0 && (face == 0 ? l < kTwK : l < kTwJ) && jl < t.ny && kl < t.nz;
    // the producer's entries of this line: level q of its sweep at src + q * kTwFace
    double* src = nb >= 0 ? (fwd ? t.exf : t.exb) + (face == 0 ? 0 : t.rows_cap / kTwFace) +
                                (size_t)__ldcg(t.rbase + nb) / kTwFace + (size_t)l
                          : nullptr;
    // the producer's levels in sweep order
    int pf = 1, pl = 0;
    if (line_ok) {
        const int lo = __ldcg(t.tlo + nb), hi = __ldcg(t.thi + nb);
        if (hi >= lo) {
            pf = fwd ? lo : nlevels - 1 - hi;
            pl = fwd ? hi : nlevels - 1 - lo;
        }
    }
    int next = line_ok ? s_first : s_last + 1;  // next level (sweep order) this lane stages
    int staged_face = -1;                       // levels of this face published so far
    const long long t0 = clock64();
    for (unsigned polls = 1;; ++polls) {
        const int mine = (int)ld_acquire_cta_sh(&sh.mine);
        const int lim = min(s_last, mine + kTwRing - 1);  // ring room
        if (next <= lim) {
            // up to kTwPoll levels: an entry per level that needs one, loaded at once
            double v[kTwPoll];
            bool need[kTwPoll];
#pragma unroll
            for (int u = 0; u < kTwPoll; ++u) {
                const int sq = next + u;
                const int L = fwd ? sq : nlevels - 1 - sq;
                const int i = L - jl - kl;
                need[u] = sq <= lim && sq - 1 >= pf && sq - 1 <= pl && i >= 0 && i < nx;
                v[u] = need[u] ? ld_relaxed_gpu_f64(src + (size_t)(sq - 1 - pf) * kTwFace) : 0.0;
            }
            int u = 0;
            for (; u < kTwPoll && next + u <= lim; ++u) {
                if (need[u] && __double_as_longlong(v[u]) == (long long)kTwEmpty) break;  // not written yet
                const int sq = next + u;
                const int L = fwd ? sq : nlevels - 1 - sq;
                const int i = L - jl - kl;
                sh.ring[face][sq % kTwRing][l] = need[u] ? v[u] : 0.0;
                if (MODE == TW_BUILD) {
                    uint8_t m = 0;
                    if (need[u]) {
                        const size_t d = ((size_t)kp * t.ny + jp) * (size_t)nx + i;
                        const uint32_t c0 = __ldcg(t.coff + d), c1 = __ldcg(t.coff + d + 1);
                        if (c1 != c0) m = (uint8_t)(__ldcg(t.icm_c + c0) >> 16);
                    }
                    sh.ringm[face][sq % kTwRing][l] = m;
                }
                if (need[u]) st_relaxed_gpu_u64(src + (size_t)(sq - 1 - pf) * kTwFace, kTwEmpty);
            }
            next += u;
        }
        // a face's levels are staged up to the least of its lanes
        int fm = next;
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) fm = min(fm, __shfl_xor_sync(0xffffffffu, fm, o));
        __syncwarp();
        if ((lane == 0 || lane == 16) && fm > staged_face) {
            st_release_cta_sh(&sh.avail[face], (unsigned long long)fm);
            staged_face = fm;
        }
        if (__all_sync(0xffffffffu, next > s_last)) break;
        if ((polls & 63u) == 0u && __shfl_sync(0xffffffffu, (int)(tw_failed(t) || clock64() - t0 > kTwWaitCycles), 0)) {
            if (lane == 0) {
                atomicOr(t.err, kTwErrWait);
                st_release_cta_sh(&sh.avail[0], ~0ull >> 1);  // release this tile's compute warps
                st_release_cta_sh(&sh.avail[1], ~0ull >> 1);
            }
            break;
        }
    }
}

// Compute-thread wait until the ring holds neighbour values for level s.
__device__ __forceinline__ void tw_wait(const TwArgs& t, TwShared& sh, int which, unsigned long long s) {
    if (ld_acquire_cta_sh(&sh.avail[which]) > s) return;
    const long long t0 = clock64();
    for (unsigned spin = 0; ld_acquire_cta_sh(&sh.avail[which]) <= s; ++spin) {
        if ((spin & 255u) == 255u && (tw_failed(t) || clock64() - t0 > kTwWaitCycles)) {
            atomicOr(t.err, kTwErrWait);
            return;
        }
    }
}

// Operands of this line's entry of the q-th level of the sweep into shared
// slot q mod kTwDepth, as one cp.async group: the (i, mask, count) word, and
// for the solves the 16-byte (r, factor) or (q, factor) record through L2 (r
// is written by other CTAs in the update phase). The row layout makes each of
// a warp's copies one contiguous stretch. Levels past the sweep's end commit
// an empty group, so every level commits exactly one.
template <int MODE>
__device__ __forceinline__ void tw_stage(const TwArgs& t, TwShared& sh, int tid, size_t e, bool live, int q) {
    if (live) {
        const int slot = q % kTwDepth;
        cp_async4(&sh.icm[slot][tid], t.icm + e);
        if (MODE != TW_BUILD) cp_async16(&sh.rec[slot][tid], (MODE == TW_FORWARD ? t.rp : t.qp) + e);
    }
    cp_commit();
}

// One tile's sweep. BUILD: the MIC(0) factor into rp.y and qp.y (forward
// order). FORWARD: q = L^-1 r into qp.x. BACKWARD: z = L^-T q, plus the z*r products in cell
// order for the reference dot order.
template <int MODE>
__device__ void tw_sweep(const TwArgs& t, TwShared& sh, int tile, int nlevels) {
    const PcgArgs& a = t.a;
    const int tid = threadIdx.x;
    const int J = tile % t.tj, K = tile / t.tj;
    constexpr bool fwd = MODE != TW_BACKWARD;
    // upstream neighbours of this sweep
    const int nby = fwd ? (J > 0 ? tile - 1 : -1) : (J + 1 < t.tj ? tile + 1 : -1);
    const int nbz = fwd ? (K > 0 ? tile - t.tj : -1) : (K + 1 < t.tk ? tile + t.tj : -1);
    const int lo = __ldcg(t.tlo + tile), hi = __ldcg(t.thi + tile);
    const int s_first = hi < lo ? nlevels : (fwd ? lo : nlevels - 1 - hi);
    const int s_last = hi < lo ? nlevels - 1 : (fwd ? hi : nlevels - 1 - lo);
    if (tid == 0) {
        sh.mine = (unsigned long long)s_first;
        sh.avail[0] = sh.avail[1] = (unsigned long long)s_first;
    }
    __syncthreads();
    if (tid >= kTwLines) {
        tw_progress_warp<MODE>(t, sh, tile, nby, nbz, s_first, s_last, nlevels);
        __syncthreads();
        return;
    }
    const int lj = tid % kTwJ, lk = tid / kTwJ;
    const int j = J * kTwJ + lj, k = K * kTwK + lk;
    const int nx = t.nx;
    const int jk = j + k;
    // This line's row entries, level q of the sweep (q = s - s_first) at
    // row0 + (fwd ? q : nlev - 1 - q) * kTwLines + tid. The operands of the
    // next kTwDepth levels are in flight to shared memory at all times: level
    // q stages q + kTwDepth, one cp.async group per level, so when level q is
    // read the group that staged it has kTwDepth - 1 groups after it.
    const int nlev = s_last - s_first + 1;
    const size_t row0 = nlev > 0 ? (size_t)__ldcg(t.rbase + tile) : 0;
    // the lines on the downstream faces write an exchange entry at every level
    // of the sweep where their cell lies in the grid (0 where the line has no
    // fluid cell), so the downstream tile's progress warp finds every entry it
    // polls written; level q's entry of face line l is ex + q * kTwFace
    double* const ex_own = (fwd ? t.exf : t.exb) + row0 / kTwFace;
    const bool in_grid = j < t.ny && k < t.nz;
    double* const ex_y = in_grid && (fwd ? lj == kTwJ - 1 : lj == 0) ? ex_own + (size_t)lk : nullptr;
    double* const ex_z = in_grid && (fwd ? lk == kTwK - 1 : lk == 0) ? ex_own + t.rows_cap / kTwFace + (size_t)lj
                                                                      : nullptr;
    auto entry = [&](int q) -> size_t {
        return row0 + (size_t)(fwd ? q : nlev - 1 - q) * kTwLines + (size_t)tid;
    };
    for (int q = 0; q < kTwDepth; ++q) tw_stage<MODE>(t, sh, tid, q < nlev ? entry(q) : 0, q < nlev, q);
    double carry = 0.0;   // the value of this line's previous cell (the -x / +x predecessor)
    uint8_t carry_m = 0;  // its neighbour mask (factorisation)
    const double TAU = 0.97, SIGMA = 0.25;
    const bool yb = fwd ? lj == 0 : lj == kTwJ - 1;  // this line reads the y neighbour tile
    const bool zb = fwd ? lk == 0 : lk == kTwK - 1;
    unsigned long long* const timing = a.timing;  // optional section timers (thread 0)
    long long t_loop = 0, t_wait = 0;
    if (timing && (tid == 0 || tid == 32)) t_loop = clock64();
    for (int s = s_first; s <= s_last; ++s) {
        const int L = fwd ? s : nlevels - 1 - s;
        const int q = s - s_first;
        const int slot = q % kTwDepth;
        cp_wait_n<kTwDepth - 1>();
        const uint32_t word = sh.icm[slot][tid];
        if (timing && tid == 0 && nby >= 0) {
            const long long w0 = clock64();
            tw_wait(t, sh, 0, (unsigned long long)s);
            t_wait += clock64() - w0;
        } else if (tid == 0 && nby >= 0) {
            tw_wait(t, sh, 0, (unsigned long long)s);
        }
        if (timing && tid == 32 && nbz >= 0) {
            const long long w0 = clock64();
            tw_wait(t, sh, 1, (unsigned long long)s);
            t_wait += clock64() - w0;
        } else if (tid == 32 && nbz >= 0) {
            tw_wait(t, sh, 1, (unsigned long long)s);
        }
        tw_bar();
        // levels before s are complete (every eighth level: the progress warp
        // only needs it to reuse ring slots, 32 levels deep)
        if (tid == 0 && ((s - s_first) & 7) == 0) st_release_cta_sh(&sh.mine, (unsigned long long)s);
        const int wp = (s - 1) & 1, wc = s & 1, rs = s % kTwRing;
        const int i = L - jk;
        const size_t ent = entry(q);
        if (word == kTwNoCell) {
            if (i >= 0 && i < nx) {  // no cell here: the downstream entry still gets written
                if (ex_y) st_relaxed_gpu_f64(ex_y + (size_t)q * kTwFace, 0.0);
                if (ex_z) st_relaxed_gpu_f64(ex_z + (size_t)q * kTwFace, 0.0);
            }
            tw_stage<MODE>(t, sh, tid, q + kTwDepth < nlev ? entry(q + kTwDepth) : 0, q + kTwDepth < nlev, q + kTwDepth);
            continue;
        }
        const uint8_t m = (uint8_t)(word >> 16);
        const double2 rec = MODE == TW_BUILD ? make_double2(0.0, 0.0) : sh.rec[slot][tid];
        const double a0 = MODE == TW_BUILD ? (double)(word >> 24) : rec.x;  // diag, r or q
        const double b0 = rec.y;                                              // the factor
        if (MODE == TW_BUILD) {
            double axi = 0, pxi = 0, axi_y = 0, axi_z = 0;
            double ayj = 0, pyj = 0, ayj_x = 0, ayj_z = 0;
            double azk = 0, pzk = 0, azk_x = 0, azk_y = 0;
            if (m >> NB_MX & 1) {
                axi = -1.0;
                pxi = carry;
                axi_y = (carry_m >> NB_PY & 1) ? -1.0 : 0.0;
                axi_z = (carry_m >> NB_PZ & 1) ? -1.0 : 0.0;
            }
            if (m >> NB_MY & 1) {
                const uint8_t mk = yb ? sh.ringm[0][rs][lk] : sh.m[wp][tid - 1];
                pyj = yb ? sh.ring[0][rs][lk] : sh.v[wp][tid - 1];
                ayj = -1.0;
                ayj_x = (mk >> NB_PX & 1) ? -1.0 : 0.0;
                ayj_z = (mk >> NB_PZ & 1) ? -1.0 : 0.0;
            }
            if (m >> NB_MZ & 1) {
                const uint8_t mk = zb ? sh.ringm[1][rs][lj] : sh.m[wp][tid - kTwJ];
                pzk = zb ? sh.ring[1][rs][lj] : sh.v[wp][tid - kTwJ];
                azk = -1.0;
                azk_x = (mk >> NB_PX & 1) ? -1.0 : 0.0;
                azk_y = (mk >> NB_PY & 1) ? -1.0 : 0.0;
            }
            const double tx = dmul(axi, pxi), ty = dmul(ayj, pyj), tz = dmul(azk, pzk);
            const double diag = a0;
            const double mx = dmul(dmul(dmul(axi, dadd(axi_y, axi_z)), pxi), pxi);
            const double my = dmul(dmul(dmul(ayj, dadd(ayj_x, ayj_z)), pyj), pyj);
            const double mz = dmul(dmul(dmul(azk, dadd(azk_x, azk_y)), pzk), pzk);
            double e = dsub(dsub(dsub(dsub(diag, dmul(tx, tx)), dmul(ty, ty)), dmul(tz, tz)),
                            dmul(TAU, dadd(dadd(mx, my), mz)));
            if (e < dmul(SIGMA, diag)) e = diag;
            const double pc = e > 0.0 ? ddiv(1.0, __dsqrt_rn(e)) : 0.0;
            t.rp[ent].y = pc;
            t.qp[ent].y = pc;
            sh.v[wc][tid] = pc;
            sh.m[wc][tid] = m;
            carry = pc;
            carry_m = m;
            if (ex_y) st_relaxed_gpu_f64(ex_y + (size_t)q * kTwFace, pc);
            if (ex_z) st_relaxed_gpu_f64(ex_z + (size_t)q * kTwFace, pc);
        } else if (MODE == TW_FORWARD) {
            // t = r + pq[-x] + pq[-y] + pq[-z]; q = t * pc (pcg_apply_mic0, forward)
            double tt = a0;
            if (m >> NB_MX & 1) tt = dadd(tt, carry);
            if (m >> NB_MY & 1) tt = dadd(tt, yb ? sh.ring[0][rs][lk] : sh.v[wp][tid - 1]);
            if (m >> NB_MZ & 1) tt = dadd(tt, zb ? sh.ring[1][rs][lj] : sh.v[wp][tid - kTwJ]);
            const double qv = dmul(tt, b0);
            const double pqv = dmul(b0, qv);
            t.qp[ent].x = qv;
            sh.v[wc][tid] = pqv;
            carry = pqv;
            if (ex_y) st_relaxed_gpu_f64(ex_y + (size_t)q * kTwFace, pqv);
            if (ex_z) st_relaxed_gpu_f64(ex_z + (size_t)q * kTwFace, pqv);
        } else {
            // t = q + pc z[+x] + pc z[+y] + pc z[+z]; z = t * pc (pcg_apply_mic0, backward)
            const double pc = b0;
            double tt = a0;
            if (m >> NB_PX & 1) tt = dadd(tt, dmul(pc, carry));
            if (m >> NB_PY & 1) tt = dadd(tt, dmul(pc, yb ? sh.ring[0][rs][lk] : sh.v[wp][tid + 1]));
            if (m >> NB_PZ & 1) tt = dadd(tt, dmul(pc, zb ? sh.ring[1][rs][lj] : sh.v[wp][tid + kTwJ]));
            const double zv = dmul(tt, pc);
            t.zr[ent] = zv;
            if (a.exact_dots)  // the reference dot order is over cells in cell order
                a.prod[__ldcg(t.coff + ((size_t)k * t.ny + j) * (size_t)nx + i)] = dmul(zv, __ldcg(&t.rp[ent].x));
            sh.v[wc][tid] = zv;
            carry = zv;
            if (ex_y) st_relaxed_gpu_f64(ex_y + (size_t)q * kTwFace, zv);
            if (ex_z) st_relaxed_gpu_f64(ex_z + (size_t)q * kTwFace, zv);
        }
        // the slot's values are in registers: it takes the level kTwDepth ahead
        tw_stage<MODE>(t, sh, tid, q + kTwDepth < nlev ? entry(q + kTwDepth) : 0, q + kTwDepth < nlev, q + kTwDepth);
    }
    cp_wait_n<0>();  // nothing in flight into the slots the next sweep reuses
    tw_bar();
    if (tid == 0) {
        if (timing && s_last >= s_first) {  // per tile: level-loop cycles, y waits, levels, sweeps
            const unsigned long long loop = (unsigned long long)(clock64() - t_loop);
            atomicAdd(timing + 9, loop);
            atomicAdd(timing + 8, (unsigned long long)t_wait);
            atomicAdd(timing + 10, (unsigned long long)(s_last - s_first + 1));
            atomicAdd(timing + 11, 1ull);
            if (nby < 0 && nbz < 0) {  // a tile that never waits: the bare level step
                atomicAdd(timing + 12, loop);
                atomicAdd(timing + 13, (unsigned long long)(s_last - s_first + 1));
            }
        }
    }
    if (timing && tid == 32 && s_last >= s_first) atomicAdd(timing + 15, (unsigned long long)t_wait);  // z waits
    __syncthreads();  // the progress warp has published the final count and left
}

// Every tile of this CTA: tiles blockIdx.x, blockIdx.x + gridDim.x, ... in
// increasing order forward (each tile after its -y and -z neighbours) and in
// decreasing order backward, so waits always point to tiles earlier in some
// CTA's order and the earliest unfinished tile can always run.
template <int MODE>
__device__ bool tw_sweep_all(const TwArgs& t, TwShared& sh, int nlevels) {
    const int G = (int)gridDim.x, b = (int)blockIdx.x;
    if (MODE == TW_BACKWARD) {
        if (b < t.ntiles)
            for (int tile = b + ((t.ntiles - 1 - b) / G) * G; tile >= 0; tile -= G) tw_sweep<MODE>(t, sh, tile, nlevels);
    } else {
        for (int tile = b; tile < t.ntiles; tile += G) tw_sweep<MODE>(t, sh, tile, nlevels);
    }
    return !tw_failed(t);
}

// ---------------------------------------------------------------- the solve
// Launched cooperatively (every CTA resident at once).
__global__ void __launch_bounds__(kTwBS, 2) k_pcg_tiles(TwArgs t) {
    __shared__ TwShared sh;
    const PcgArgs& a = t.a;
    const uint32_t nf = *a.nf;
    const uint32_t ntile = (nf + kTile - 1) / kTile;
    const uint32_t G = gridDim.x * kTwBS, gt = blockIdx.x * kTwBS + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * kTwWarps + (threadIdx.x >> 5), nw = gridDim.x * kTwWarps;
    const int nlevels = a.nlevels;
    int parity = 0;
    double residual = 0.0, sigma = 0.0;
    // phase timers of CTA 0 (between grid barriers every CTA passes together)
    const bool timed = a.timing != nullptr && blockIdx.x == 0 && threadIdx.x == 0;
    long long tck = timed ? clock64() : 0;
#define TW_SECTION(idx)                                              \
    do {                                                             \
        if (timed) {                                                 \
            const long long now_ = clock64();                        \
            atomicAdd(a.timing + (idx), (unsigned long long)(now_ - tck)); \
            tck = now_;                                              \
        }                                                            \
    } while (0)
    int iters = 0;
    double mx = 0.0;
    for (uint32_t i = gt; i < nf; i += G) mx = fmax(mx, fabs(a.b[i]));
    for (uint32_t q = gt; q < (uint32_t)t.ntiles; q += G) {
        t.tlo[q] = INT32_MAX;
        t.thi[q] = -1;
    }
    if (!tw_grid_max(t, sh, mx, parity, residual)) goto out;
    if (residual > a.tol) {
        // r and p, the cell-order words, and the tiles' level ranges
        for (uint32_t i = gt; i < nf; i += G) {
            const uint32_t cell = a.lv_cell[i];
            const int ii = (int)(cell % (uint32_t)t.nx), jj = (int)((cell / (uint32_t)t.nx) % (uint32_t)t.ny),
                      kk = (int)(cell / ((uint32_t)t.nx * (uint32_t)t.ny));
            t.icm_c[a.cinv[i]] = (uint32_t)ii | (uint32_t)a.nmask[i] << 16 | (uint32_t)a.diag[i] << 24;
            a.r[i] = a.b[i];
            a.p[i] = 0.0;
            const int tile = jj / kTwJ + (kk / kTwK) * t.tj;
            atomicMin(t.tlo + tile, ii + jj + kk);
            atomicMax(t.thi + tile, ii + jj + kk);
        }
        if (!tw_grid_sync(t, sh)) goto out;
        // each tile's first row entry: a prefix over the tiles' level counts (one warp)
        if (blockIdx.x == 0 && threadIdx.x < 32) {
            unsigned long long run = 0;
            for (int b0 = 0; b0 < t.ntiles; b0 += 32) {
                const int q = b0 + lane;
                unsigned long long n = 0;
                if (q < t.ntiles) {
                    const int lo = __ldcg(t.tlo + q), hi = __ldcg(t.thi + q);
                    n = hi >= lo ? (unsigned long long)(hi - lo + 1) * kTwLines : 0ull;
                }
                unsigned long long x = n;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
                    if (lane >= o) x += y;
                }
                if (q < t.ntiles) t.rbase[q] = (uint32_t)(run + x - n);
                run += __shfl_sync(0xffffffffu, x, 31);
            }
            if (lane == 0) {
                t.rbase[t.ntiles] = (uint32_t)min(run, (unsigned long long)t.rows_cap);
                if (run > (unsigned long long)t.rows_cap) atomicOr(t.err, kTwErrWait);  // cannot happen: sized per tile
            }
        }
        if (!tw_grid_sync(t, sh)) goto out;
        {  // rows: every entry without a cell, then every cell's entry; every exchange entry unwritten
            const size_t nrow = __ldcg(t.rbase + t.ntiles);
            for (size_t q = gt; q < nrow; q += G) t.icm[q] = kTwNoCell;
            const size_t nex = nrow / kTwFace, xf = t.rows_cap / kTwFace;
            unsigned long long* ef = reinterpret_cast<unsigned long long*>(t.exf);
            unsigned long long* eb = reinterpret_cast<unsigned long long*>(t.exb);
            for (size_t q = gt; q < nex; q += G) {
                ef[q] = kTwEmpty;
                ef[xf + q] = kTwEmpty;
                eb[q] = kTwEmpty;
                eb[xf + q] = kTwEmpty;
            }
        }
        if (!tw_grid_sync(t, sh)) goto out;
        for (uint32_t i = gt; i < nf; i += G) {
            const uint32_t cell = a.lv_cell[i];
            const int ii = (int)(cell % (uint32_t)t.nx), jj = (int)((cell / (uint32_t)t.nx) % (uint32_t)t.ny),
                      kk = (int)(cell / ((uint32_t)t.nx * (uint32_t)t.ny));
            const int tile = jj / kTwJ + (kk / kTwK) * t.tj;
            const size_t e = (size_t)__ldcg(t.rbase + tile) +
                             (size_t)(ii + jj + kk - __ldcg(t.tlo + tile)) * kTwLines +
                             (size_t)((kk % kTwK) * kTwJ + jj % kTwJ);
            if (e >= t.rows_cap) continue;  // cannot happen: the ranges were sized above
            t.icm[e] = (uint32_t)ii | (uint32_t)a.nmask[i] << 16 | (uint32_t)a.diag[i] << 24;
            t.rp[e].x = a.b[i];
            t.tpos[i] = (uint32_t)e;
        }
        if (!tw_grid_sync(t, sh)) goto out;
        if (!tw_sweep_all<TW_BUILD>(t, sh, nlevels)) goto out;
        if (!tw_grid_sync(t, sh)) goto out;  // the factor's exchange planes are reused by the sweeps
        TW_SECTION(0);
        if (!tw_sweep_all<TW_FORWARD>(t, sh, nlevels)) goto out;
        if (!tw_sweep_all<TW_BACKWARD>(t, sh, nlevels)) goto out;
        // dot(z, r)
        if (a.exact_dots) {
            if (!tw_exact_dot(t, sh, sigma)) goto out;
        } else {
            if (!tw_grid_sync(t, sh)) goto out;
            for (uint32_t tl = (uint32_t)gw; tl < ntile; tl += (uint32_t)nw) {
                double acc = 0.0;
                const uint32_t e = min((tl + 1) * kTile, nf);
                for (uint32_t i = tl * kTile + lane; i < e; i += 32)
                    acc = dadd(acc, dmul(__ldcg(t.zr + t.tpos[i]), __ldcg(a.r + i)));
                acc = warp_tree_sum(acc);
                if (lane == 0) a.tpart[tl] = acc;
            }
            if (!tw_grid_sync(t, sh)) goto out;
            sigma = tw_tile_total(t, ntile, sh);
        }
        for (uint32_t i = gt; i < nf; i += G) a.s[i] = __ldcg(t.zr + t.tpos[i]);
        if (!tw_grid_sync(t, sh)) goto out;
        for (int it = 0; it < a.max_iters; ++it) {
            iters = it + 1;
            // apply_a (pressure.rs:400-439) and s*As, by the tiles of the tree dot
            for (uint32_t tl = (uint32_t)gw; tl < ntile; tl += (uint32_t)nw) {
                double acc = 0.0;
                for (int u = 0; u < kTile / 32; ++u) {
                    const uint32_t i = tl * kTile + lane + 32u * u;
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
                    if (lane == 0) a.tpart[tl] = acc;
                }
            }
            double denom;  // dot(s, As)
            if (a.exact_dots) {
                if (!tw_exact_dot(t, sh, denom)) goto out;
            } else {
                if (!tw_grid_sync(t, sh)) goto out;
                denom = tw_tile_total(t, ntile, sh);
            }
            TW_SECTION(3);
            if (fabs(denom) < 1e-30) break;
            const double alpha = ddiv(sigma, denom);
            double mr = 0.0;
            for (uint32_t i = gt; i < nf; i += G) {
                a.p[i] = dadd(a.p[i], dmul(alpha, __ldcg(a.s + i)));
                const double rv = dsub(a.r[i], dmul(alpha, __ldcg(a.as + i)));
                a.r[i] = rv;
                t.rp[t.tpos[i]].x = rv;
                mr = fmax(mr, fabs(rv));
            }
            if (!tw_grid_max(t, sh, mr, parity, residual)) goto out;  // also publishes r and rp.x
            TW_SECTION(5);
            if (residual <= a.tol) break;
            if (!tw_sweep_all<TW_FORWARD>(t, sh, nlevels)) goto out;
            if (!tw_sweep_all<TW_BACKWARD>(t, sh, nlevels)) goto out;
            double sigma_new;  // dot(z, r)
            if (a.exact_dots) {
                if (!tw_exact_dot(t, sh, sigma_new)) goto out;
            } else {
                if (!tw_grid_sync(t, sh)) goto out;
                for (uint32_t tl = (uint32_t)gw; tl < ntile; tl += (uint32_t)nw) {
                    double acc = 0.0;
                    const uint32_t e = min((tl + 1) * kTile, nf);
                    for (uint32_t i = tl * kTile + lane; i < e; i += 32)
                        acc = dadd(acc, dmul(__ldcg(t.zr + t.tpos[i]), __ldcg(a.r + i)));
                    acc = warp_tree_sum(acc);
                    if (lane == 0) a.tpart[tl] = acc;
                }
                if (!tw_grid_sync(t, sh)) goto out;
                TW_SECTION(1);  // the sweeps end at this barrier
                sigma_new = tw_tile_total(t, ntile, sh);
            }
            const double beta = ddiv(sigma_new, sigma);
            for (uint32_t i = gt; i < nf; i += G) a.s[i] = dadd(__ldcg(t.zr + t.tpos[i]), dmul(beta, a.s[i]));
            if (!tw_grid_sync(t, sh)) goto out;  // s complete before the next matvec reads neighbours
            TW_SECTION(6);
            sigma = sigma_new;
        }
        for (uint32_t i = gt; i < nf; i += G) a.p_dense[a.lv_cell[i]] = a.p[i];
    }
out:
    TW_SECTION(7);
#undef TW_SECTION
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *a.out_iters = iters;
        *a.out_residual = residual;
        if (a.timing) a.timing[14] += 1;
    }
}

}  // namespace sdr
