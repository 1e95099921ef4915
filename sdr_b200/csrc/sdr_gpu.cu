// sdr_gpu.cu — host orchestration and C ABI of the B200 FLIP/PIC substep.
//
// One sdr_solver owns a CUDA stream, the device-resident grid/particle/solve
// state and a pinned status block. Solver::step's CFL loop and the emission
// RNG stay on the host in f64 (they are sequential and tiny); every other
// phase of Solver::substep is a kernel. After each substep one small status
// copy returns the particle count, counters and the face maxima that the
// next cfl_dt needs.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <new>
#include <string>
#include <vector>

#include "sdr_gpu.h"
#include "common.cuh"
#include "grid.cuh"
#include "metrics.cuh"
#include "particles.cuh"
#include "pressure.cuh"
#include "pressure_cluster.cuh"
#include "pressure_tiles.cuh"
#include "render.cuh"
#include "scan.cuh"
#include "sdf.cuh"
#include "packed.cuh"

using namespace sdr;

namespace {

thread_local std::string g_err;
std::atomic<uint64_t> g_launches{0};
// sdr_debug_inject: the fault the next matching call on this thread injects.
thread_local int g_fault = 0;
// Set by a packed batch engine around sdr_solver_create: the new solver runs
// on the engine's stream instead of a stream of its own.
thread_local cudaStream_t g_engine_stream = nullptr;

struct Fail {
    int code;
    std::string msg;
};

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            throw Fail{e_ == cudaErrorMemoryAllocation ? SDR_ERR_OOM : SDR_ERR_CUDA,      \
                       std::string(#call) + ": " + cudaGetErrorString(e_)};               \
    } while (0)

#define LAUNCH(kern, grid, block, smem, stream, ...)                    \
    do {                                                                \
        kern<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);       \
        g_launches.fetch_add(1, std::memory_order_relaxed);             \
        CK(cudaGetLastError());                                         \
    } while (0)

// A substep kernel through sdr_solver::issue (launched, or recorded while
// packing); the call site's line keys its slot in a packed launch.
#define SLAUNCH(kern, grid, block, smem, stream, ...) issue<kern##_op>(kern, __LINE__, (grid), (block), (smem), __VA_ARGS__)
#define MSET(p, v, bytes) mset(__LINE__, (p), (v), (bytes))
#define MCOPY(d, s, bytes) mcopy(__LINE__, (d), (s), (bytes))

inline unsigned blocks(size_t n, unsigned bs) { return (unsigned)std::max<size_t>(1, (n + bs - 1) / bs); }

// Fluid cells from which SDR_PCG_AUTO solves on a cluster instead of one block
// (the fluid count of the previous solve decides).
constexpr uint32_t kClusterMinFluidCells = 200000;

// CTAs in the cluster of a one-cluster kernel, once per device and kernel:
// 16 (one per SM, the largest non-portable cluster) when the device can
// schedule it for that kernel, else the portable 8.
template <class Kern>
int cluster_ctas(Kern kernel, int slot, int threads, int device, size_t dyn_smem = 0) {
    static std::mutex mu;
    static int ctas[3][64] = {};
    if (device < 0 || device >= 64) throw Fail{SDR_ERR_CUDA, "device index out of range"};
    std::lock_guard<std::mutex> lk(mu);
    if (!ctas[slot][device]) {
        int n = dyn_smem ? 4 : 8;  // without an answer: a size every GPC holds
        if (cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
            cudaLaunchConfig_t cfg{};
            cfg.gridDim = dim3(kClMaxCtas);
            cfg.blockDim = dim3(threads);
            cfg.dynamicSmemBytes = dyn_smem;
            int mx = 0;
            if (cudaOccupancyMaxPotentialClusterSize(&mx, kernel, &cfg) == cudaSuccess && mx >= 1) {
                n = 1;
                while (n * 2 <= mx && n * 2 <= kClMaxCtas) n *= 2;  // largest power of two it allows
            }
        }
        cudaGetLastError();  // a refused query leaves the default
        ctas[slot][device] = n;
    }
    return ctas[slot][device];
}

// Launch a kernel as exactly one cluster of `ctas` CTAs on `st`.
template <class Kern, class... Args>
void launch_one_cluster_smem(Kern kernel, int ctas, int threads, size_t dyn_smem, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)ctas);
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = dyn_smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)ctas;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, kernel, args...));
    g_launches.fetch_add(1, std::memory_order_relaxed);
}

template <class Kern, class... Args>
void launch_one_cluster(Kern kernel, int ctas, int threads, cudaStream_t st, Args... args) {
    launch_one_cluster_smem(kernel, ctas, threads, 0, st, args...);
}

// Solver-owned device buffers come from one library memory pool per device,
// allocated and released in the order of the owning solver's stream
// (cudaMallocFromPoolAsync / cudaFreeAsync). Unlike cudaMalloc/cudaFree this
// neither synchronises the device nor takes the driver's allocation lock for
// long, so one scene's set-up, growth or teardown does not stall the scenes
// running beside it; a freed block is reused by the next scene without a
// round trip to the driver. The pool keeps up to a quarter of device memory
// cached between scenes and returns the rest at synchronisation points.
cudaMemPool_t device_pool() {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw Fail{SDR_ERR_CUDA, "device index out of range"};
    std::lock_guard<std::mutex> lk(mu);
    if (!pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        CK(cudaMemPoolCreate(&pool, &props));
        size_t free_b = 0, total_b = 0;
        CK(cudaMemGetInfo(&free_b, &total_b));
        uint64_t keep = total_b / 4;
        CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        pools[dev] = pool;
    }
    return pools[dev];
}

// Without a stream (one-shot entry points) these are plain cudaMalloc/cudaFree.
template <class T>
void dalloc(T*& p, size_t n, cudaStream_t s = nullptr) {
    if (p) {
        if (s) cudaFreeAsync(p, s);
        else cudaFree(p);
    }
    p = nullptr;
    size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
    if (s) CK(cudaMallocFromPoolAsync((void**)&p, bytes, device_pool(), s));
    else CK(cudaMalloc((void**)&p, bytes));
}

template <class T>
void dfree(T*& p, cudaStream_t s = nullptr) {
    if (p) {
        if (s) cudaFreeAsync(p, s);
        else cudaFree(p);
    }
    p = nullptr;
}

// Pinned host blocks (status words, emission staging, frame buffers) come
// from a process-wide cache of power-of-two blocks: cudaFreeHost synchronises
// the device, so a block is never handed back to the driver, only to the
// cache, which is bounded by the peak number of blocks in use at once.
class PinnedCache {
   public:
    static void* get(size_t bytes, size_t* granted = nullptr) {
        int cls = size_class(bytes);
        size_t size = (size_t)1 << cls;
        if (granted) *granted = size;
        {
            std::lock_guard<std::mutex> lk(mu());
            auto& fl = lists()[cls];
            if (!fl.empty()) {
                void* p = fl.back();
                fl.pop_back();
                return p;
            }
        }
        void* p = nullptr;
        CK(cudaMallocHost(&p, size));
        return p;
    }
    static void put(void* p, size_t bytes) {
        if (!p) return;
        std::lock_guard<std::mutex> lk(mu());
        lists()[size_class(bytes)].push_back(p);
    }

   private:
    static int size_class(size_t bytes) {
        int c = 8;  // 256-byte minimum
        while (((size_t)1 << c) < bytes) ++c;
        return c;
    }
    static std::mutex& mu() {
        static std::mutex m;
        return m;
    }
    static std::vector<void*>* lists() {
        static std::vector<void*> l[64];
        return l;
    }
};

template <class T>
void hget(T*& p, size_t n, size_t* granted_elems = nullptr) {
    size_t g = 0;
    p = static_cast<T*>(PinnedCache::get(std::max<size_t>(n, 1) * sizeof(T), &g));
    if (granted_elems) *granted_elems = g / sizeof(T);
}

// `n` must be the element count the block was requested (or granted) with.
template <class T>
void hput(T*& p, size_t n) {
    PinnedCache::put(p, std::max<size_t>(n, 1) * sizeof(T));
    p = nullptr;
}

// Device scalars returned to the host after every substep.
struct DevStatus {
    uint32_t n;             // particle count
    uint32_t err;           // device-side error bits
    unsigned int maxbits[3];
    int iters;
    double residual;
    unsigned long long drained, culled, moves;
    uint32_t nf;            // fluid cells of the last solve
    uint32_t ncand;
    uint32_t nmoves;
    uint32_t long_count;
    uint32_t p2g_queue;     // P2G nodes with particles this substep
    uint32_t total;         // scratch scan total
    uint32_t hist_max;
    unsigned long long fluid_count;
    unsigned long long wall_count;
    unsigned long long pcg_cycles[16];
    unsigned long long redist_cand, redist_sweeps, redist_long;  // cumulative
    unsigned long long redist_rounds;                            // cumulative
};

__device__ __forceinline__ void k_set_u32_body(VB, uint32_t* p, uint32_t v) {
    if (threadIdx.x == 0) *p = v;
}
__global__ void k_set_u32(uint32_t* p, uint32_t v) { k_set_u32_body(VB{blockIdx.x, gridDim.x}, p, v); }
__device__ __forceinline__ void k_redist_begin_body(VB, RedistState* r) {
    if (threadIdx.x != 0) return;
    r->ncand = 0;
    r->active = 1;
    r->nmoves = 0;
    r->par = 0;
    r->nmoves_par = 0;
    r->err = 0;
}
__global__ void k_redist_begin(RedistState* r) { k_redist_begin_body(VB{blockIdx.x, gridDim.x}, r); }
__device__ __forceinline__ void k_redist_end_body(VB, const RedistState* r, DevStatus* s) {
    if (threadIdx.x != 0) return;
    s->moves = r->moves_total;
    s->err |= r->err;
    s->redist_cand = r->cand_total;
    s->redist_sweeps = r->sweeps_total;
    s->redist_long = r->long_total;
    s->redist_rounds = r->rounds_total;
}
__global__ void k_redist_end(const RedistState* r, DevStatus* s) { k_redist_end_body(VB{blockIdx.x, gridDim.x}, r, s); }

// The kernels of a substep as packable operations (largest block of their call sites).
SDR_OP(k_set_u32, 32)
SDR_OP(k_scan_tiles, kScanBS)
SDR_OP(k_scan_sums, kScanBS)
SDR_OP(k_scan_apply, kScanBS)
SDR_OP(k_cavity_and_base, 256)
SDR_OP(k_base_labels, 256)
SDR_OP(k_classify_keys, kBS)
SDR_OP(k_sort_scatter, kBS)
SDR_OP(k_sort_segments, 256)
SDR_OP(k_sort_long, 256)
SDR_OP(k_sorted_records, kBS)
SDR_OP(k_p2g_nodes, kBS)
SDR_OP(k_p2g, kBS)
SDR_OP(k_add_forces, 256)
SDR_OP(k_enforce_solid, 256)
SDR_OP(k_lines_count, 256)
SDR_OP(k_lines_assign, 256)
SDR_OP(k_level_starts_dev, 256)
SDR_OP(k_tables, 256)
SDR_OP(k_fluid_flags, 256)
SDR_OP(k_corder, 256)
SDR_OP(k_pcg, kPcgBS)
SDR_OP(k_gradient, 256)
SDR_OP(k_extrap_valid, 256)
SDR_OP(k_extrap, 256)
SDR_OP(k_face_max, 256)
SDR_OP(k_g2p_advect, kBS)
SDR_OP(k_bounds_flags, kBS)
SDR_OP(k_compact, kBS)
SDR_OP(k_redist_begin, 32)
SDR_OP(k_redist_hist_n, kBS)
SDR_OP(k_redist_append, kBS)
SDR_OP(k_redist_replay, kRedistBS)
SDR_OP(k_redist_par, kRpBS)
SDR_OP(k_redist_end, 32)
__global__ void k_f64_to_f32(const double* __restrict__ in, float* __restrict__ out, size_t n) {
    size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) out[q] = (float)in[q];
}
__global__ void k_pack_particles(const double* __restrict__ xyz, float4* __restrict__ out, size_t n) {
    size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) out[q] = make_float4((float)xyz[3 * q], (float)xyz[3 * q + 1], (float)xyz[3 * q + 2], 0.f);
}

// xorshift64 (solver.rs:120-140).
inline uint64_t rng_next(uint64_t& s) {
    uint64_t x = s;
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    s = x;
    return x;
}
inline double rng_unit(uint64_t& s) { return (double)(rng_next(s) >> 11) / (double)(1ULL << 53); }

struct V3 {
    double x, y, z;
};
inline V3 vadd(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 vmul(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 vcross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double vlen(V3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
inline V3 vnorm0(V3 a) {  // math.rs:73-80
    double l = vlen(a);
    if (l > 1e-12) return {a.x / l, a.y / l, a.z / l};
    return {0, 0, 0};
}

}  // namespace

struct sdr_solver {
    int device = 0;
    cudaStream_t st = nullptr;
    bool own_stream = true;   // false: the stream belongs to a packed batch engine
    Packer* pk = nullptr;     // set: operations are recorded for a packed launch instead of issued
    std::vector<sdr_metrics*> collectors;  // live metrics collectors of this solver
    Grid g{};
    size_t ncell = 0, nu = 0, nv = 0, nw = 0;
    int snx = 0, sny = 0, snz = 0;
    double sdx = 0, sox = 0, soy = 0, soz = 0;
    // parameters
    sdr_fluid_params fluid{};
    sdr_needle needle{};
    bool has_outlet = false;
    Aabb outlet{};
    uint64_t max_iters = 200;
    double tol = 1e-6;
    // scalar state (solver.rs:155-179)
    double time = 0.0, emit_accum = 0.0, last_residual = 0.0;
    uint64_t steps = 0, last_pcg_iters = 0, last_substeps = 0, drained = 0;
    uint64_t rng = 0x5deece66dULL | 1ULL;
    uint64_t emitted = 0, culled = 0, redistributed = 0;
    uint32_t n = 0;
    size_t cap = 0;
    double grid_speed = 0.0;  // MacGrid::max_speed of the current faces
    // device state
    double* sdf64 = nullptr;
    float* sdf32 = nullptr;
    float *u = nullptr, *v = nullptr, *w = nullptr, *su = nullptr, *sv = nullptr, *sw = nullptr;
    uint8_t *ku = nullptr, *kv = nullptr, *kw = nullptr;  // extrapolation: when each face became known
    uint8_t *cells = nullptr, *base = nullptr, *cavity = nullptr;
    float4 *pos = nullptr, *vel = nullptr, *pos2 = nullptr, *vel2 = nullptr;
    int* key_cell = nullptr;
    uint32_t *key_sort = nullptr, *perm = nullptr, *ptmp = nullptr, *flag = nullptr, *off = nullptr;
    uint32_t *drn = nullptr;
    uint32_t *hist_valid = nullptr, *hist_sort = nullptr, *start = nullptr, *fill = nullptr;
    uint32_t* long_list = nullptr;
    double4* lrec = nullptr;
    float4* vrec = nullptr;
    uint32_t* tsum = nullptr;
    size_t tsum_cap = 0;
    DevStatus* dst = nullptr;
    DevStatus* hst = nullptr;  // pinned
    // pressure
    int nlevels = 0, nchunks = 0;
    uint32_t *lines_cnt = nullptr, *lv_cell = nullptr, *cflag = nullptr, *coff = nullptr;
    int *level_start = nullptr, *pos_of_cell = nullptr, *nbr = nullptr, *corder = nullptr,
        *chunk_start = nullptr, *cinv = nullptr;
    uint8_t *diag = nullptr, *nmask = nullptr;
    double *b = nullptr, *precon = nullptr, *p = nullptr, *r = nullptr, *z = nullptr, *s = nullptr,
           *as = nullptr, *q = nullptr, *pq = nullptr, *partials = nullptr, *p_dense = nullptr, *prod = nullptr;
    int4 *frec = nullptr, *brec = nullptr;
    // redistribution
    uint32_t* cand = nullptr;
    uint32_t* rpend = nullptr;  // 2 x cand_n: pending units of the long-list rounds
    uint32_t* rbits = nullptr;  // particle-index bitmap of the long-list sort: (capacity + 31) / 32 words
    size_t cand_n = 0;      // entries of `cand`
    size_t cand_limit = 0;  // sdr_solver_set_candidate_capacity (0: the particle capacity)
    uint32_t* moves = nullptr;
    RedistState* rds = nullptr;
    // emission staging (pinned)
    float4* h_epos = nullptr;
    float4* h_evel = nullptr;
    size_t h_ecap = 0;
    // metrics scratch
    CellPart* mcell = nullptr;
    double* mpart = nullptr;
    size_t mpart_cap = 0;
    MetricsOut* mout = nullptr;
    MetricsOut* h_mout = nullptr;
    bool sorted_valid = false;  // perm/start describe the current particle set
    unsigned long long redist_seen[4] = {0, 0, 0, 0};  // device redistribution counters at the last status read
    // long candidate lists decided over every SM (k_redist_par_grid), set up on first use
    int rp_grid = 0;                // CTAs of its cooperative launch (0: not set up, -1: unavailable)
    double* rp_slots = nullptr;
    unsigned* rp_bar = nullptr;
    // timing
    cudaEvent_t ev[10] = {};
    cudaEvent_t ev_block = nullptr;  // blocking-sync event (SDR_SOLVER_BLOCKING_SYNC)
    bool profiling = false;
    bool kernel_timers = false;  // profiling level 2: section timers inside k_pcg
    bool exact_dots = false;  // reference dot order in the PCG (bit-exact pressure)
    int pcg_kernel = SDR_PCG_AUTO;  // which pressure-solve kernel (SDR_PCG_*)
    int pcg_ctas = 0;               // CTAs of k_pcg's cluster (0: 1 on a shared GPU, else the device's largest)
    bool shared_gpu = false;        // SDR_SOLVER_SHARED_GPU
    int ctas_pcg = 0, ctas_pcgc = 0, ctas_rp = 0;  // largest clusters the device schedules (asked once)
    double* tpart = nullptr;        // tile sums of the tree-order dots
    uint32_t* p2g_list = nullptr;   // grid nodes with particles around them (P2G queue)
    uint32_t last_p2g_queue = 0;    // its length at the last status read
    uint32_t last_nf = 0;           // fluid cells of the last solve (picks the kernel under SDR_PCG_AUTO)
    double* cl_slots = nullptr;     // CTA partials of the cluster kernels
    // whole-GPU tiled solve (k_pcg_tiles), allocated on first use
    uint32_t *tw_icm = nullptr, *tw_icm_c = nullptr, *tw_tpos = nullptr, *tw_rbase = nullptr;
    double2 *tw_rp = nullptr, *tw_qp = nullptr;
    size_t tw_rows = 0;  // row entries of the sweeps' operand rows
    double *tw_z = nullptr, *tw_exf = nullptr, *tw_exb = nullptr,
           *tw_slots = nullptr;
    int *tw_lo = nullptr, *tw_hi = nullptr;
    unsigned* tw_bar = nullptr;
    int tw_tj = 0, tw_tk = 0, tw_grid = 0;  // tiles along y and z; CTAs of the cooperative launch (0: not set up)
    unsigned long long* rclaim = nullptr;  // per cell: claim stamps of the parallel redistribution replay
    sdr_profile prof{};
    uint64_t particle_substeps = 0, substeps_total = 0;
    double device_ms = 0.0;

    // A kernel of the substep: launched on the solver's stream, or recorded
    // for the packed launch while a Packer is attached.
    template <class Op, class Kern, class... A>
    void issue(Kern kern, int line, unsigned grid, unsigned block, size_t smem, A... args) {
        if (pk) {
            pk->record<Op>(line, grid, block, smem, args...);
            return;
        }
        kern<<<grid, block, smem, st>>>(args...);
        g_launches.fetch_add(1, std::memory_order_relaxed);
        CK(cudaGetLastError());
    }
    void mset(int line, void* p, int v, size_t bytes) {
        if (!bytes) return;
        if (pk) {
            pk->record<k_pack_memset_op>(line, (unsigned)((bytes + kPackChunk - 1) / kPackChunk), 256, 0,
                                         static_cast<unsigned char*>(p), v, bytes);
            return;
        }
        CK(cudaMemsetAsync(p, v, bytes, st));
    }
    // Device-to-device, or host-to-device from pinned staging.
    void mcopy(int line, void* d, const void* s, size_t bytes) {
        if (!bytes) return;
        if (pk) {
            pk->record<k_pack_copy_op>(line, (unsigned)((bytes + kPackChunk - 1) / kPackChunk), 256, 0,
                                       static_cast<unsigned char*>(d), static_cast<const unsigned char*>(s), bytes);
            return;
        }
        CK(cudaMemcpyAsync(d, s, bytes, cudaMemcpyDefault, st));
    }

    void create_events() {
        for (auto& e : ev) CK(cudaEventCreate(&e));
    }
    void mark(int i) {
        if (!pk && (profiling || i == 0 || i == 9)) CK(cudaEventRecord(ev[i], st));
    }
    float elapsed(int a, int b) const {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev[a], ev[b]);
        return ms;
    }

    double particle_volume() const {  // solver.rs:225-228
        double cell = g.dx * g.dx * g.dx;
        return cell / (double)std::max<uint64_t>(fluid.particles_per_cell, 1);
    }
    double jet_speed() const {  // solver.rs:107-114
        double area = M_PI * needle.radius * needle.radius;
        return area > 0.0 ? needle.flow_rate / area : 0.0;
    }
    Sdf sdf_f() const { return Sdf{snx, sny, snz, (float)sdx, (float)sox, (float)soy, (float)soz, sdf32}; }
    SdfD sdf_d() const { return SdfD{snx, sny, snz, sdx, sox, soy, soz, sdf64}; }
    Faces faces() const { return Faces{u, v, w}; }
    size_t nnodes() const { return ((size_t)g.nx + 1) * ((size_t)g.ny + 1) * ((size_t)g.nz + 1); }
    Faces saved() const { return Faces{su, sv, sw}; }
    uint32_t* dn() { return &dst->n; }

    // Exclusive scan; `site` (the caller's line) keys its kernels in a packed launch.
    void scan(const uint32_t* in, uint32_t* out, size_t n_, uint32_t* total, int site) {
        const int key = 1000000 + 4 * site;
        if (n_ == 0) {
            if (total) issue<k_set_u32_op>(k_set_u32, key, 1, 1, 0, total, 0u);
            return;
        }
        uint32_t nt = (uint32_t)((n_ + kScanTile - 1) / kScanTile);
        if (nt > tsum_cap) {
            dalloc(tsum, nt, st);
            tsum_cap = nt;
        }
        issue<k_scan_tiles_op>(k_scan_tiles, key + 1, nt, kScanBS, 0, in, (uint32_t)n_, tsum);
        issue<k_scan_sums_op>(k_scan_sums, key + 2, 1, kScanBS, 0, tsum, nt, total);
        issue<k_scan_apply_op>(k_scan_apply, key + 3, nt, kScanBS, 0, in, (uint32_t)n_, tsum, out);
    }

    void ensure_capacity(size_t need) {
        if (need <= cap) return;
        size_t ncap = std::max(need + need / 2, cap + cap / 2);
        ncap = std::max<size_t>(ncap, 256);
        // Stream-ordered: the copies run after every queued use of the old
        // arrays and the old arrays are released after the copies.
        float4 *np = nullptr, *nv_ = nullptr;
        dalloc(np, ncap, st);
        dalloc(nv_, ncap, st);
        if (n) {
            CK(cudaMemcpyAsync(np, pos, (size_t)n * sizeof(float4), cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(nv_, vel, (size_t)n * sizeof(float4), cudaMemcpyDeviceToDevice, st));
        }
        dfree(pos, st);
        dfree(vel, st);
        pos = np;
        vel = nv_;
        dalloc(pos2, ncap, st);
        dalloc(vel2, ncap, st);
        dalloc(key_cell, ncap, st);
        dalloc(key_sort, ncap, st);
        dalloc(perm, ncap, st);
        dalloc(ptmp, ncap, st);
        dalloc(flag, ncap + 1, st);
        dalloc(off, ncap + 1, st);
        dalloc(drn, ncap, st);
        cand_n = cand_limit ? std::min(ncap, cand_limit) : ncap;
        dalloc(cand, cand_n, st);
        dalloc(rpend, 2 * cand_n, st);
        dalloc(rbits, (ncap + 31) / 32 + 1, st);
        dalloc(moves, ncap * 2, st);
        dalloc(lrec, ncap, st);
        dalloc(vrec, ncap, st);
        cap = ncap;
        sorted_valid = false;
    }

    void alloc_grid() {
        size_t nc = ncell;
        dalloc(u, nu, st); dalloc(v, nv, st); dalloc(w, nw, st);
        dalloc(su, nu, st); dalloc(sv, nv, st); dalloc(sw, nw, st);
        dalloc(p2g_list, nnodes(), st);
        dalloc(ku, nu, st); dalloc(kv, nv, st); dalloc(kw, nw, st);
        CK(cudaMemsetAsync(u, 0, nu * 4, st));
        CK(cudaMemsetAsync(v, 0, nv * 4, st));
        CK(cudaMemsetAsync(w, 0, nw * 4, st));
        CK(cudaMemsetAsync(su, 0, nu * 4, st));
        CK(cudaMemsetAsync(sv, 0, nv * 4, st));
        CK(cudaMemsetAsync(sw, 0, nw * 4, st));
        dalloc(cells, nc, st); dalloc(base, nc, st); dalloc(cavity, nc, st);
        CK(cudaMemsetAsync(cells, AIR, nc, st));
        dalloc(hist_valid, nc + 1, st);
        dalloc(hist_sort, nc + 1, st);
        dalloc(start, nc + 1, st);
        dalloc(fill, nc + 1, st);
        dalloc(long_list, nc, st);
        nlevels = g.nx + g.ny + g.nz - 2;
        nchunks = (int)((nc + kDotChunk - 1) / kDotChunk);
        dalloc(lines_cnt, (size_t)nlevels * g.nz + 1, st);
        dalloc(level_start, nlevels + 1, st);
        dalloc(pos_of_cell, nc, st);
        dalloc(lv_cell, nc, st);
        dalloc(nbr, nc * 6, st);
        dalloc(diag, nc, st);
        dalloc(nmask, nc, st);
        dalloc(b, nc, st); dalloc(precon, nc, st); dalloc(p, nc, st); dalloc(r, nc, st); dalloc(z, nc, st);
        dalloc(s, nc, st); dalloc(as, nc, st); dalloc(q, nc, st); dalloc(pq, nc, st);
        dalloc(partials, nchunks + 1, st);
        if (!cl_slots) dalloc(cl_slots, 2 * kClMaxCtas, st);
        dalloc(tpart, ncell / kTile + 2, st);
        dalloc(rclaim, ncell, st);
        CK(cudaMemsetAsync(rclaim, 0, ncell * sizeof(unsigned long long), st));
        dalloc(corder, nc, st);
        dalloc(cinv, nc, st);
        dalloc(prod, nc, st);
        dalloc(frec, nc, st);
        dalloc(brec, nc, st);
        dalloc(chunk_start, nchunks + 1, st);
        dalloc(cflag, nc + 1, st);
        dalloc(coff, nc + 1, st);
        CK(cudaMemsetAsync(cflag + nc, 0, 4, st));  // coff[nc] = the fluid count (line ends of the tiled solve)
        dalloc(p_dense, nc, st);
        CK(cudaMemsetAsync(p_dense, 0, nc * 8, st));
        dalloc(mcell, blocks(nc, kMetBS), st);
        dalloc(mout, 1, st);
    }

    void free_all() {
        dfree(sdf64, st); dfree(sdf32, st);
        dfree(u, st); dfree(v, st); dfree(w, st); dfree(su, st); dfree(sv, st); dfree(sw, st);
        dfree(ku, st); dfree(kv, st); dfree(kw, st);
        dfree(cells, st); dfree(base, st); dfree(cavity, st);
        dfree(pos, st); dfree(vel, st); dfree(pos2, st); dfree(vel2, st);
        dfree(key_cell, st); dfree(key_sort, st); dfree(perm, st); dfree(ptmp, st); dfree(flag, st); dfree(off, st); dfree(drn, st);
        dfree(hist_valid, st); dfree(hist_sort, st); dfree(start, st); dfree(fill, st); dfree(long_list, st); dfree(tsum, st);
        dfree(dst, st);
        dfree(lines_cnt, st); dfree(lv_cell, st); dfree(cflag, st); dfree(coff, st); dfree(level_start, st); dfree(pos_of_cell, st);
        dfree(nbr, st); dfree(corder, st); dfree(cinv, st); dfree(prod, st); dfree(frec, st); dfree(brec, st); dfree(chunk_start, st); dfree(diag, st); dfree(nmask, st);
        dfree(b, st); dfree(precon, st); dfree(p, st); dfree(r, st); dfree(z, st); dfree(s, st); dfree(as, st); dfree(q, st); dfree(pq, st);
        dfree(tw_icm, st); dfree(tw_icm_c, st); dfree(tw_tpos, st); dfree(tw_rbase, st); dfree(tw_rp, st); dfree(tw_qp, st); dfree(tw_z, st); dfree(tw_exf, st); dfree(tw_exb, st); dfree(tw_slots, st); dfree(tw_lo, st);
        dfree(tw_hi, st); dfree(tw_bar, st);
        dfree(rp_slots, st); dfree(rp_bar, st);
        dfree(partials, st); dfree(p_dense, st); dfree(cl_slots, st); dfree(rclaim, st); dfree(tpart, st); dfree(p2g_list, st);
        dfree(cand, st); dfree(rpend, st); dfree(rbits, st); dfree(moves, st); dfree(rds, st); dfree(lrec, st); dfree(vrec, st);
        dfree(mcell, st); dfree(mpart, st); dfree(mout, st);
        if (hst) hput(hst, 1);
        if (h_epos) hput(h_epos, h_ecap);
        if (h_evel) hput(h_evel, h_ecap);
        if (h_mout) hput(h_mout, 1);
        h_ecap = 0;
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        if (ev_block) cudaEventDestroy(ev_block);
        ev_block = nullptr;
        if (st && own_stream) cudaStreamDestroy(st);
        st = nullptr;
    }

    void refresh_base() {
        SLAUNCH(k_cavity_and_base, blocks(ncell, 256), 256, 0, st, g, sdf_d(), (int)has_outlet, outlet,
               cavity, base, 0);
    }

    // ---------------------------------------------------------------- phases
    void emit(double dt) {  // solver.rs:313-339
        double pv = particle_volume();
        if (pv <= 0.0 || needle.flow_rate <= 0.0 || time >= needle.inject_until) return;
        emit_accum += needle.flow_rate * dt / pv;
        double count = std::floor(emit_accum);
        size_t k = (size_t)count;
        emit_accum -= count;
        if (k == 0) return;
        ensure_capacity((size_t)n + k);
        if (k > h_ecap) {
            CK(cudaStreamSynchronize(st));
            if (h_epos) hput(h_epos, h_ecap);
            if (h_evel) hput(h_evel, h_ecap);
            h_ecap = 0;
            size_t c = std::max<size_t>(k * 2, 4096);
            hget(h_epos, c, &c);
            hget(h_evel, c);
            h_ecap = c;
        }
        V3 axis = vnorm0({needle.axis.x, needle.axis.y, needle.axis.z});
        V3 a = std::fabs(axis.x) < 0.9 ? V3{1, 0, 0} : V3{0, 1, 0};  // solver.rs:933-942
        V3 e1 = vnorm0(vcross(axis, a));
        V3 e2 = vnorm0(vcross(axis, e1));
        V3 vv = vmul(axis, jet_speed());
        V3 tip{needle.tip.x, needle.tip.y, needle.tip.z};
        for (size_t i = 0; i < k; ++i) {
            double rr = needle.radius * std::sqrt(rng_unit(rng));
            double th = 2.0 * M_PI * rng_unit(rng);
            double along = (rng_unit(rng) - 0.5) * g.dx;
            V3 ps = vadd(vadd(vadd(tip, vmul(e1, rr * std::cos(th))), vmul(e2, rr * std::sin(th))),
                         vmul(axis, along));
            h_epos[i] = make_float4((float)ps.x, (float)ps.y, (float)ps.z, 0.f);
            h_evel[i] = make_float4((float)vv.x, (float)vv.y, (float)vv.z, 0.f);
        }
        MCOPY(pos + n, h_epos, k * sizeof(float4));
        MCOPY(vel + n, h_evel, k * sizeof(float4));
        if (profiling) prof.h2d_bytes += 2 * k * sizeof(float4);
        // The staging buffers are reused next substep; the status sync at the
        // end of this substep orders the copies before any reuse.
        n += (uint32_t)k;
        emitted += k;
        SLAUNCH(k_set_u32, 1, 1, 0, st, dn(), n);
        sorted_valid = false;
    }

    void classify(bool mark) {
        MSET(hist_valid, 0, (ncell + 1) * 4);
        MSET(hist_sort, 0, (ncell + 1) * 4);
        if (mark) SLAUNCH(k_base_labels, blocks(ncell, 256), 256, 0, st, base, cells, ncell);
        if (n)
            SLAUNCH(k_classify_keys, blocks(n, kBS), kBS, 0, st, g, pos, n, (int)has_outlet, outlet,
                   (int)mark, cells, key_cell, key_sort, hist_valid, hist_sort);
    }

    void sort() {  // counting sort by the f32 P2G cell key
        scan(hist_sort, start, ncell + 1, &dst->total, __LINE__);
        MCOPY(fill, start, ncell * 4);
        if (n) SLAUNCH(k_sort_scatter, blocks(n, kBS), kBS, 0, st, key_sort, n, fill, perm);
        MSET(&dst->long_count, 0, 4);
        SLAUNCH(k_sort_segments, blocks(ncell, 256), 256, 0, st, start, (uint32_t)ncell, perm, long_list,
               &dst->long_count);
        SLAUNCH(k_sort_long, 148, 256, 0, st, start, long_list, &dst->long_count, perm, ptmp);
        if (n) SLAUNCH(k_sorted_records, blocks(n, kBS), kBS, 0, st, g, pos, vel, perm, n, lrec, vrec);
        sorted_valid = true;
    }

    void p2g(double dt, bool fused) {
        P2GArgs a{};
        a.g = g;
        a.lrec = lrec;
        a.vrec = vrec;
        a.start = start;
        a.u = u; a.v = v; a.w = w;
        a.su = su; a.sv = sv; a.sw = sw;
        a.cells = cells;
        a.gdt[0] = fluid.gravity.x * dt;
        a.gdt[1] = fluid.gravity.y * dt;
        a.gdt[2] = fluid.gravity.z * dt;
        a.add_forces = fused;
        a.enforce = fused;
        // empty nodes at once, the rest queued for the eight-lane gather; its grid
        // follows the last queue length (the loop over the queue covers any length)
        MSET(&dst->p2g_queue, 0, 4);
        SLAUNCH(k_p2g_nodes, blocks(nnodes(), kBS), kBS, 0, st, a, p2g_list, &dst->p2g_queue);
        const size_t want = last_p2g_queue ? ((size_t)last_p2g_queue + last_p2g_queue / 4 + 64) * kP2GLanes
                                           : nnodes() * kP2GLanes;  // no history yet: every node
        SLAUNCH(k_p2g, (unsigned)std::min<size_t>(blocks(want, kBS), 148 * 16), kBS, 0, st, a, p2g_list,
               &dst->p2g_queue);
    }

    void add_forces(double dt) {  // solver.rs:593-604
        if (fluid.gravity.x != 0.0) SLAUNCH(k_add_forces, blocks(nu, 256), 256, 0, st, u, nu, fluid.gravity.x * dt);
        if (fluid.gravity.y != 0.0) SLAUNCH(k_add_forces, blocks(nv, 256), 256, 0, st, v, nv, fluid.gravity.y * dt);
        if (fluid.gravity.z != 0.0) SLAUNCH(k_add_forces, blocks(nw, 256), 256, 0, st, w, nw, fluid.gravity.z * dt);
    }

    void project(double dt, bool enforce) {  // pressure.rs:123-239 + solver.rs:290-300
        project_setup(dt, enforce);
        project_solve(dt);
        project_gradient(dt);
    }

    // enforce_solid_faces, wavefront numbering, neighbour tables, RHS, dot chunks.
    void project_setup(double dt, bool enforce) {
        unsigned ngrid = blocks(nnodes(), 256);
        if (enforce) SLAUNCH(k_enforce_solid, ngrid, 256, 0, st, g, cells, u, v, w);
        size_t nl = (size_t)nlevels * g.nz;
        SLAUNCH(k_lines_count, blocks(nl, 256), 256, 0, st, g, cells, nlevels, lines_cnt);
        MSET(lines_cnt + nl, 0, 4);
        scan(lines_cnt, lines_cnt, nl + 1, &dst->nf, __LINE__);
        SLAUNCH(k_lines_assign, blocks(nl, 256), 256, 0, st, g, cells, nlevels, lines_cnt, pos_of_cell, lv_cell);
        SLAUNCH(k_level_starts_dev, blocks(nlevels + 1, 256), 256, 0, st, lines_cnt, nlevels, g.nz, &dst->nf,
               level_start);
        TableArgs t{};
        t.g = g;
        t.cells = cells;
        t.pos_of_cell = pos_of_cell;
        t.lv_cell = lv_cell;
        t.nf = &dst->nf;
        t.nbr = nbr;
        t.diag = diag;
        t.nmask = nmask;
        t.b = b;
        t.u = u; t.v = v; t.w = w;
        t.hist = hist_valid;
        t.inv_scale = fluid.density * g.dx / dt;
        double k_vol = fluid.volume_stiffness;
        t.vs_on = (k_vol > 0.0 && dt > 0.0) ? 1 : 0;
        t.vs_rest = (double)std::max<uint64_t>(fluid.particles_per_cell, 1);
        t.vs_k = k_vol;
        t.vs_unit = g.dx / dt;
        t.vs_cap = 0.25 * t.vs_unit;
        SLAUNCH(k_tables, blocks(ncell, 256), 256, 0, st, t);
        SLAUNCH(k_fluid_flags, blocks(ncell, 256), 256, 0, st, cells, ncell, cflag);
        scan(cflag, coff, ncell + 1, nullptr, __LINE__);
        SLAUNCH(k_corder, blocks(ncell, 256), 256, 0, st, cells, ncell, coff, pos_of_cell, corder, cinv, chunk_start,
               nchunks, &dst->nf);
        MSET(p_dense, 0, ncell * 8);
    }

    void project_solve(double dt) {
        (void)dt;
        PcgArgs a{};
        a.nf = &dst->nf;
        a.nlevels = nlevels;
        a.nchunks = nchunks;
        a.nx = g.nx;
        a.ny = g.ny;
        a.frec = frec;
        a.brec = brec;
        a.level_start = level_start;
        a.nbr = nbr;
        a.diag = diag;
        a.nmask = nmask;
        a.corder = corder;
        a.cinv = cinv;
        a.prod = prod;
        a.chunk_start = chunk_start;
        a.b = b;
        a.precon = precon; a.p = p; a.r = r; a.z = z; a.s = s; a.as = as; a.q = q; a.pq = pq;
        a.partials = partials;
        a.tpart = tpart;
        a.slots = cl_slots;
        a.tol = tol;
        a.max_iters = (int)std::min<uint64_t>(max_iters, (uint64_t)INT32_MAX);
        a.lv_cell = lv_cell;
        a.p_dense = p_dense;
        a.out_iters = &dst->iters;
        a.out_residual = &dst->residual;
        a.timing = kernel_timers ? dst->pcg_cycles : nullptr;
        a.exact_dots = exact_dots ? 1 : 0;
        if (pk) {  // packed with other scenes: one block per scene, a plain (recordable) launch
            SLAUNCH(k_pcg, 1, kPcgBS, kPcgSmem, st, a);
            return;
        }
        // fluid cells of the last solve; before the first one, the cells the
        // particles fill at particles_per_cell each
        const uint64_t nf_hint =
            last_nf ? (uint64_t)last_nf : (uint64_t)n / std::max<uint64_t>(fluid.particles_per_cell, 1);
        const bool large = pcg_kernel == SDR_PCG_AUTO && nf_hint >= kClusterMinFluidCells && !shared_gpu;
        if ((pcg_kernel == SDR_PCG_TILES || large) && tiles_ready()) {
            launch_tiles(a);
            if (profiling) prof.pcg_tile_launches += 1;
            return;
        }
        const bool cluster = pcg_kernel == SDR_PCG_CLUSTER || pcg_kernel == SDR_PCG_TILES || large ||
                             (pcg_kernel == SDR_PCG_AUTO && nf_hint >= kClusterMinFluidCells);
        if (cluster) {
            // One cluster of up to 16 CTAs (one per SM); the levels of each
            // sweep are separated by the hardware cluster barrier.
            a.timing = nullptr;
            if (!ctas_pcgc) ctas_pcgc = cluster_ctas(k_pcg_cluster, 0, kClBS, device);
            launch_one_cluster(k_pcg_cluster, ctas_pcgc, kClBS, st, a);
            if (profiling) prof.pcg_cluster_launches += 1;
        } else {
            // Sweeps on CTA 0, elementwise phases on the whole cluster: one
            // CTA when the GPU is shared with other scenes (each solve then
            // holds one SM), else the largest cluster the device schedules.
            // 8 CTAs measured best on the real cavity (1: 2202, 4: 2039, 8: 2024,
            // 16: 2060 ms of solve over three frames): past 8 the cluster barrier
            // costs more than the extra bandwidth gives
            int ctas = 1;
            if (pcg_ctas > 0 || !shared_gpu) {
                if (!ctas_pcg) ctas_pcg = cluster_ctas(k_pcg, 2, kPcgBS, device, kPcgSmem);
                ctas = pcg_ctas > 0 ? std::min(pcg_ctas, ctas_pcg) : std::min(ctas_pcg, 8);
            }
            if (ctas == 1) {
                // a plain launch: the kernel sees a cluster of one CTA, and the
                // launch overlaps other streams' kernels like any other
                SLAUNCH(k_pcg, 1, kPcgBS, kPcgSmem, st, a);
            } else {
                launch_one_cluster_smem(k_pcg, ctas, kPcgBS, kPcgSmem, st, a);
            }
        }
    }

    // Cooperative launch of k_redist_par_grid (every CTA resident): false if
    // the device cannot run it (then the cluster decides long lists).
    bool rounds_grid_ready() {
        if (rp_grid != 0) return rp_grid > 0;
        int coop = 0, nsm = 0, occ = 0;
        CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
        CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_redist_par_grid, kRpBS, 0) != cudaSuccess) {
            cudaGetLastError();
            occ = 0;
        }
        if (!coop || occ < 1) {
            rp_grid = -1;
            return false;
        }
        rp_grid = nsm * std::min(occ, 2);
        dalloc(rp_slots, 2 * (size_t)rp_grid, st);
        dalloc(rp_bar, 2, st);
        return true;
    }

    // The whole-GPU tiled solve needs a cooperative launch with every CTA
    // resident; its buffers are allocated on first use. False if the device
    // cannot run it (then the cluster kernel solves).
    bool tiles_ready() {
        if (tw_grid < 0) return false;
        if (tw_grid > 0) return true;
        int coop = 0, nsm = 0, occ = 0;
        CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
        CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_pcg_tiles, kTwBS, 0) != cudaSuccess) {
            cudaGetLastError();
            occ = 0;
        }
        if (!coop || occ < 1 || g.nx > INT16_MAX) {  // the sweeps keep i in 16 bits
            tw_grid = -1;
            return false;
        }
        tw_grid = nsm * std::min(occ, 2);
        tw_tj = (g.ny + kTwJ - 1) / kTwJ;
        tw_tk = (g.nz + kTwK - 1) / kTwK;
        const size_t nt = (size_t)tw_tj * tw_tk;
        // operand rows: a tile's levels span at most nx + kTwJ + kTwK - 2 of them
        tw_rows = nt * (size_t)(g.nx + kTwJ + kTwK) * (size_t)kTwLines;
        if (tw_rows >= (size_t)UINT32_MAX) {  // row entries are 32-bit
            tw_grid = -1;
            return false;
        }
        dalloc(tw_icm, tw_rows, st); dalloc(tw_rp, tw_rows, st); dalloc(tw_qp, tw_rows, st); dalloc(tw_z, tw_rows, st);
        dalloc(tw_icm_c, ncell, st); dalloc(tw_tpos, ncell, st); dalloc(tw_rbase, nt + 1, st);
        // exchange planes: two faces of one entry per line and row level
        dalloc(tw_exf, 2 * (tw_rows / kTwFace), st); dalloc(tw_exb, 2 * (tw_rows / kTwFace), st);
        dalloc(tw_lo, nt, st); dalloc(tw_hi, nt, st);
        dalloc(tw_bar, 2, st);
        dalloc(tw_slots, 2 * (size_t)tw_grid, st);
        return true;
    }

    void launch_tiles(const PcgArgs& a) {
        TwArgs t{};
        t.a = a;  // a.timing: the section timers of profiling level 2
        t.nx = g.nx; t.ny = g.ny; t.nz = g.nz;
        t.tj = tw_tj; t.tk = tw_tk; t.ntiles = tw_tj * tw_tk;
        t.coff = coff;
        t.icm = tw_icm; t.rp = tw_rp; t.qp = tw_qp; t.zr = tw_z;
        t.icm_c = tw_icm_c; t.tpos = tw_tpos; t.rbase = tw_rbase; t.rows_cap = tw_rows;
        t.exf = tw_exf; t.exb = tw_exb;
        t.tlo = tw_lo; t.thi = tw_hi;
        t.bar = tw_bar;
        t.gslots = tw_slots;
        t.err = &dst->err;
        CK(cudaMemsetAsync(tw_bar, 0, 2 * sizeof(unsigned), st));  // a wound-down launch may leave arrivals
        void* args[] = {&t};
        CK(cudaLaunchCooperativeKernel((const void*)k_pcg_tiles, dim3((unsigned)tw_grid), dim3(kTwBS), args, 0, st));
        g_launches.fetch_add(1, std::memory_order_relaxed);
    }

    void project_gradient(double dt) {
        unsigned ngrid = blocks(nnodes(), 256);
        double coef = dt / (fluid.density * g.dx);
        SLAUNCH(k_gradient, ngrid, 256, 0, st, g, cells, p_dense, coef, u, v, w);
    }

    void extrapolate() {  // solver.rs:608-647
        unsigned ngrid = blocks(nnodes(), 256);
        SLAUNCH(k_extrap_valid, ngrid, 256, 0, st, g, cells, ku, kv, kw);
        MSET(dst->maxbits, 0, sizeof(dst->maxbits));
        for (int it = 0; it < 4; ++it) {  // four sweeps, in place
            ExtrapArgs e{g, u, v, w, ku, kv, kw, it, it == 3 ? dst->maxbits : nullptr};
            SLAUNCH(k_extrap, ngrid, 256, 0, st, e);
        }
    }

    void face_max() {
        MSET(dst->maxbits, 0, sizeof(dst->maxbits));
        SLAUNCH(k_face_max, 296, 256, 0, st, u, nu, &dst->maxbits[0]);
        SLAUNCH(k_face_max, 296, 256, 0, st, v, nv, &dst->maxbits[1]);
        SLAUNCH(k_face_max, 296, 256, 0, st, w, nw, &dst->maxbits[2]);
    }

    MoveArgs move_args(double dt) {
        MoveArgs a{};
        a.g = g;
        a.sdf = sdf_f();
        a.pos = pos;
        a.vel = vel;
        a.order = nullptr;
        a.n = n;
        a.f = faces();
        a.saved = saved();
        a.flip = (float)std::min(1.0, std::max(0.0, fluid.flip_ratio));
        a.dt = (float)dt;
        double bmx[3] = {sox + (double)(snx - 1) * sdx, soy + (double)(sny - 1) * sdx, soz + (double)(snz - 1) * sdx};
        a.bb = Aabb{{sox, soy, soz}, {bmx[0], bmx[1], bmx[2]}};
        a.has_outlet = has_outlet;
        a.outlet = outlet;
        a.cull_phi = (float)(0.5 * sdx);
        a.keep = flag;
        a.drained = drn;
        return a;
    }

    void g2p_advect(double dt, bool g2p_on, bool advect_on, bool bounds_on, bool use_order) {
        if (!n) return;
        MoveArgs a = move_args(dt);
        a.order = use_order && sorted_valid ? perm : nullptr;
        a.do_g2p = g2p_on;
        a.do_advect = advect_on;
        a.do_bounds = bounds_on;
        SLAUNCH(k_g2p_advect, blocks(n, kBS), kBS, 0, st, a);
    }

    void compact(bool flags_ready) {  // solver.rs:736-755
        if (!n) return;
        if (!flags_ready) {
            MoveArgs a = move_args(0.0);
            SLAUNCH(k_bounds_flags, blocks(n, kBS), kBS, 0, st, a);
        }
        scan(flag, off, n, dn(), __LINE__);
        SLAUNCH(k_compact, blocks(n, kBS), kBS, 0, st, pos, vel, flag, drn, off, n, pos2, vel2, &dst->drained);
        std::swap(pos, pos2);
        std::swap(vel, vel2);
        sorted_valid = false;
    }

    void redistribute(uint32_t n_upper) {  // solver.rs:454-557
        if (!n_upper) return;
        uint32_t cap_ = (uint32_t)std::ceil(std::max(fluid.redist_cap_factor, 1.0) *
                                             (double)std::max<uint64_t>(fluid.particles_per_cell, 1));
        V3 gd = vnorm0({fluid.gravity.x, fluid.gravity.y, fluid.gravity.z});
        RedistArgs ra{};
        ra.g = g;
        ra.sdf = sdf_f();
        ra.f = faces();
        ra.pos = pos;
        ra.vel = vel;
        ra.key_cell = key_cell;
        ra.count = hist_valid;
        ra.cavity = cavity;
        ra.cand = cand;
        ra.cand_cap = (uint32_t)cand_n;
        ra.n_upper = n_upper;
        ra.claim = rclaim;
        ra.rounds = shared_gpu ? 0 : 1;  // many scenes: spend no SM time on rounds
        ra.slots = cl_slots;
        ra.pend = rpend;
        ra.bits = rbits;
        // A GPU of its own: long lists over every SM. On a shared GPU one CTA:
        // a cluster launch waits for a whole GPC of free SMs, which other
        // scenes' solves rarely leave.
        const bool grid_rounds = !shared_gpu && !pk && rounds_grid_ready();
        if (!shared_gpu && !ctas_rp) ctas_rp = cluster_ctas(k_redist_par, 1, kRpBS, device);
        const int rp_ctas = shared_gpu ? 1 : ctas_rp;
        ra.cap = cap_;
        const double dirs[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
        for (int d = 0; d < 6; ++d) ra.down[d] = dirs[d][0] * gd.x + dirs[d][1] * gd.y + dirs[d][2] * gd.z;
        ra.moves = moves;
        ra.rs = rds;
        SLAUNCH(k_redist_begin, 1, 1, 0, st, rds);
        for (int sweep = 0; sweep < 4; ++sweep) {
            MSET(hist_valid, 0, ncell * 4);
            SLAUNCH(k_redist_hist_n, blocks(n_upper, kBS), kBS, 0, st, g, pos, dn(), rds, key_cell, hist_valid);
            SLAUNCH(k_redist_append, blocks(n_upper, kBS), kBS, 0, st, g, key_cell, hist_valid, cavity, dn(), cap_, rds, cand,
                   (uint32_t)cand_n);
            SLAUNCH(k_redist_replay, 1, kRedistBS, kRedistSmem, st, ra);
            // long lists only (the replay kernel hands over through the state; otherwise it returns at once)
            if (grid_rounds) {
                // every SM decides the long list (a cooperative launch; it returns at once for short lists)
                CK(cudaMemsetAsync(rp_bar, 0, 2 * sizeof(unsigned), st));
                double* sl = rp_slots;
                unsigned* br = rp_bar;
                void* args[] = {&ra, &sl, &br};
                CK(cudaLaunchCooperativeKernel((const void*)k_redist_par_grid, dim3((unsigned)rp_grid), dim3(kRpBS),
                                               args, 0, st));
                g_launches.fetch_add(1, std::memory_order_relaxed);
            } else if (rp_ctas == 1) {
                SLAUNCH(k_redist_par, 1, kRpBS, 0, st, ra);
            } else {
                launch_one_cluster(k_redist_par, rp_ctas, kRpBS, st, ra);
            }
        }
        SLAUNCH(k_redist_end, 1, 1, 0, st, rds, dst);
        sorted_valid = false;
    }

    // The status block back to the host (recorded while packing).
    void status_issue() {
        MCOPY(hst, dst, sizeof(DevStatus));
        if (profiling) prof.d2h_bytes += sizeof(DevStatus);
    }
    void sync_status() {
        status_issue();
        if (ev_block) {  // the waiting thread sleeps instead of spinning
            CK(cudaEventRecord(ev_block, st));
            CK(cudaEventSynchronize(ev_block));
        } else {
            CK(cudaStreamSynchronize(st));
        }
        status_read();
    }
    void status_read() {
        n = hst->n;
        drained = hst->drained;
        culled = hst->culled;
        redistributed = hst->moves;
        if (const uint32_t e = hst->err) {
            // Reported once: the error words start clean for the next call.
            // The substep that set them did not finish its redistribution.
            CK(cudaMemsetAsync(&dst->err, 0, sizeof(uint32_t), st));
            CK(cudaMemsetAsync(&rds->err, 0, sizeof(uint32_t), st));
            CK(cudaStreamSynchronize(st));
            if (e & 1u)
                throw Fail{SDR_ERR_CAPACITY, "redistribution candidate list overflow (error bits " + std::to_string(e) +
                                                 "); raise it with sdr_solver_set_candidate_capacity"};
            throw Fail{SDR_ERR_DEVICE_TIMEOUT, "a bounded device loop gave up (error bits " + std::to_string(e) + ")"};
        }
    }

    void read_grid_speed() {
        float mu, mv, mw;
        std::memcpy(&mu, &hst->maxbits[0], 4);
        std::memcpy(&mv, &hst->maxbits[1], 4);
        std::memcpy(&mw, &hst->maxbits[2], 4);
        double a = mu, b_ = mv, c = mw;
        grid_speed = std::sqrt(a * a + b_ * b_ + c * c);  // grid.rs:202-206
    }

    void substep(double dt) {  // solver.rs:284-310
        substep_issue(dt);
        sync_status();
        substep_finish(dt);
    }

    uint32_t pending_n_before = 0;  // particles the substep in flight advanced
    bool pending_timed = false;     // its start and end events were recorded

    // Every operation of one substep, on the stream or into the Packer.
    void substep_issue(double dt) {
        pending_timed = pk == nullptr;
        mark(0);
        emit(dt);
        classify(true);
        sort();
        mark(1);
        p2g(dt, true);
        mark(2);
        project_setup(dt, false);
        mark(3);
        project_solve(dt);
        mark(4);
        project_gradient(dt);
        extrapolate();
        mark(5);
        g2p_advect(dt, true, true, true, true);
        mark(6);
        uint32_t n_before = n;
        pending_n_before = n_before;
        compact(true);
        mark(7);
        if (fluid.redistribute) redistribute(n_before);
        mark(8);
        mark(9);
    }

    // Bookkeeping once the substep's status block is on the host.
    void substep_finish(double dt) {
        const uint32_t n_before = pending_n_before;
        last_pcg_iters = (uint64_t)hst->iters;
        last_residual = hst->residual;
        last_nf = hst->nf;
        last_p2g_queue = hst->p2g_queue;
        read_grid_speed();
        if (pending_timed) device_ms += elapsed(0, 9);
        particle_substeps += n_before;
        substeps_total += 1;
        if (profiling && pending_timed) {
            prof.emit_classify_sort_ms += elapsed(0, 1);
            prof.p2g_ms += elapsed(1, 2);
            prof.pressure_setup_ms += elapsed(2, 3);
            prof.pcg_ms += elapsed(3, 4);
            prof.gradient_extrapolate_ms += elapsed(4, 5);
            prof.g2p_advect_ms += elapsed(5, 6);
            prof.compact_ms += elapsed(6, 7);
            prof.redistribute_ms += elapsed(7, 8);
            prof.substeps += 1;
            prof.pcg_launches += 1;
            prof.pcg_cell_iters += (uint64_t)hst->nf * (uint64_t)std::max(hst->iters, 0);
            prof.fluid_cells += hst->nf;
            prof.particles += n_before;
            for (int q = 0; q < 16; ++q) prof.pcg_section_cycles[q] = hst->pcg_cycles[q];
        }
        account_redistribution();
        time += dt;
        steps += 1;
    }

    // Device redistribution counters since the last status read, into the profile.
    void account_redistribution() {
        if (profiling) {
            prof.redist_candidates += hst->redist_cand - redist_seen[0];
            prof.redist_sweeps += hst->redist_sweeps - redist_seen[1];
            prof.redist_long_sweeps += hst->redist_long - redist_seen[2];
            prof.redist_rounds += hst->redist_rounds - redist_seen[3];
        }
        redist_seen[0] = hst->redist_cand;
        redist_seen[1] = hst->redist_sweeps;
        redist_seen[2] = hst->redist_long;
        redist_seen[3] = hst->redist_rounds;
    }

    double cfl_dt() const {  // solver.rs:262-281
        double jet = time < needle.inject_until ? jet_speed() : 0.0;
        double gl = std::sqrt(fluid.gravity.x * fluid.gravity.x + fluid.gravity.y * fluid.gravity.y +
                              fluid.gravity.z * fluid.gravity.z);
        double gg = std::sqrt(gl * g.dx);
        double speed = std::fmax(std::fmax(std::fmax(grid_speed, jet), gg), 1e-6);
        return std::fmin(g.dx / speed, 0.01);
    }

    void step(double dt) {  // solver.rs:237-259
        const uint32_t MAX_SUBSTEPS = 512;
        double floor_ = dt / (double)MAX_SUBSTEPS;
        double remaining = dt;
        uint32_t taken = 0;
        while (remaining > 1e-12) {
            double sub = std::fmin(std::fmax(cfl_dt(), floor_), remaining);
            substep(sub);
            remaining -= sub;
            ++taken;
        }
        last_substeps = taken;
    }

    void run_phase(int ph, double dt) {
        switch (ph) {
            case SDR_PHASE_EMIT: emit(dt); break;
            case SDR_PHASE_CLASSIFY: classify(true); break;
            case SDR_PHASE_P2G:
                classify(false);
                sort();
                p2g(dt, false);
                break;
            case SDR_PHASE_ADD_FORCES: add_forces(dt); break;
            case SDR_PHASE_PROJECT:
                classify(false);  // refresh the per-cell counts of the volume source
                project(dt, true);
                break;
            case SDR_PHASE_EXTRAPOLATE: extrapolate(); break;
            case SDR_PHASE_G2P: g2p_advect(dt, true, false, false, false); break;
            case SDR_PHASE_ADVECT: g2p_advect(dt, false, true, false, false); break;
            case SDR_PHASE_BOUNDS: compact(false); break;
            case SDR_PHASE_REDISTRIBUTE:
                if (fluid.redistribute) redistribute(n);
                break;
            case SDR_PHASE_CLOCK:
                time += dt;
                steps += 1;
                break;
            default: throw Fail{SDR_ERR_INVALID, "unknown phase"};
        }
        if (ph != SDR_PHASE_CLOCK) {
            sync_status();
            if (ph == SDR_PHASE_PROJECT) {
                last_pcg_iters = (uint64_t)hst->iters;
                last_residual = hst->residual;
                last_nf = hst->nf;
                if (profiling)
                    for (int q = 0; q < 16; ++q) prof.pcg_section_cycles[q] = hst->pcg_cycles[q];
            }
            if (ph == SDR_PHASE_EXTRAPOLATE) read_grid_speed();
            if (ph == SDR_PHASE_REDISTRIBUTE) account_redistribution();
            if (ph == SDR_PHASE_P2G) last_p2g_queue = hst->p2g_queue;
        }
    }
};

struct sdr_metrics {
    sdr_solver* owner = nullptr;  // null once the solver is destroyed
    double cavity_volume = 0;
    uint8_t *is_wall = nullptr, *washed = nullptr, *wet = nullptr;
    uint64_t wall_count = 0;
    std::vector<sdr_frame_metrics> history;
    double injected_ml = 0.0;

    // Device masks are released on the owning solver's stream, whichever of
    // the two is destroyed first; the summary and history stay readable.
    void release() {
        if (!owner) return;
        dfree(is_wall, owner->st);
        dfree(washed, owner->st);
        dfree(wet, owner->st);
        auto& c = owner->collectors;
        c.erase(std::remove(c.begin(), c.end(), this), c.end());
        owner = nullptr;
    }
};

// ---------------------------------------------------------------- helpers
namespace {

template <class F>
int guard(F&& f) {
    try {
        f();
        g_err.clear();
        return SDR_OK;
    } catch (const Fail& e) {
        g_err = e.msg;
        return e.code;
    } catch (const std::bad_alloc&) {
        g_err = "host allocation failed";
        return SDR_ERR_OOM;
    } catch (...) {
        g_err = "unknown error";
        return SDR_ERR_CUDA;
    }
}

void require(bool c, const char* msg) {
    if (!c) throw Fail{SDR_ERR_INVALID, msg};
}

// Node count of an SDF grid, checked before any copy or launch: every axis
// 1..2^31-1 nodes (the kernels take int dimensions) and at most 2^37 nodes in
// all (one thread per node on a one-dimensional grid of 128-thread blocks).
size_t sdf_node_count(const uint64_t dims[3]) {
    for (int c = 0; c < 3; ++c) require(dims[c] >= 1 && dims[c] <= (uint64_t)INT32_MAX, "dims must be 1..2^31-1");
    const unsigned __int128 nn = (unsigned __int128)dims[0] * dims[1] * dims[2];
    require(nn <= ((unsigned __int128)1 << 37), "SDF grid too large (more than 2^37 nodes)");
    return (size_t)nn;
}

struct DeviceScope {
    int prev = -1;
    explicit DeviceScope(int dev) {
        cudaGetDevice(&prev);
        if (dev >= 0 && dev != prev) CK(cudaSetDevice(dev));
    }
    ~DeviceScope() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

void check_device() {
    int nd = 0;
    cudaError_t e = cudaGetDeviceCount(&nd);
    if (e != cudaSuccess || nd == 0)
        throw Fail{SDR_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e)};
}

}  // namespace

// ---------------------------------------------------------------- no-allocation SDF build
// Scratch of sdr_sdf_from_mesh_noalloc: the triangles padded to whole
// bulk-copy tiles, followed by one error word. It is a file-scope device
// array, so every GPU that loads this library holds it until exit, and every
// call on a device shares it.
namespace {
constexpr size_t kNoAllocTris = ((size_t)SDR_NOALLOC_MAX_TRIANGLES + kSdfTile - 1) / kSdfTile * kSdfTile;
constexpr size_t kNoAllocDoubles = kNoAllocTris * 9 + 2;
}  // namespace
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

namespace {
std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[128] = {};

// Device address of the scratch on the current device. In host code the
// symbol is only a host-side stand-in, so the address is looked up once per
// device with that device current, and cached.
double* noalloc_scratch() {
    int dev = -1;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 128) throw Fail{SDR_ERR_NO_DEVICE, "device ordinal out of range"};
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void* ptr = nullptr;
        CK(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
        g_noalloc_ptr[dev] = ptr;
    }
    return static_cast<double*>(g_noalloc_ptr[dev]);
}
}  // namespace

// ================================================================= C ABI
// Library-internal (not part of the C ABI): lets the host-side batch and
// serving layer report its own failures through sdr_last_error.
void sdr_internal_set_error(const std::string& msg) { g_err = msg; }

// Pixel primitives (render.cpp).
void sdr_internal_draw_disk(uint8_t* rgb, uint32_t w, uint32_t h, int64_t cx, int64_t cy, int64_t r,
                            const uint8_t c[3]);
void sdr_internal_draw_line(uint8_t* rgb, uint32_t w, uint32_t h, int64_t x0, int64_t y0, int64_t x1, int64_t y1,
                            const uint8_t c[3]);

// Metrics files (output.cpp).
std::string sdr_internal_frames_json(const sdr_frame_metrics* frames, size_t n);
std::string sdr_internal_frames_csv(const sdr_frame_metrics* frames, size_t n);
int sdr_internal_write_text(const char* path, const std::string& t, std::string& err);

extern "C" {

int sdr_abi_version(void) { return SDR_ABI_VERSION; }
const char* sdr_last_error(void) { return g_err.c_str(); }
uint64_t sdr_kernel_launch_count(void) { return g_launches.load(); }

int sdr_solver_create(const sdr_sdf_desc* sdf, double sim_dx, const sdr_fluid_params* fluid,
                      const sdr_needle* needle, const sdr_solver_options* options, sdr_solver** out) {
    return guard([&] {
        require(sdf && fluid && needle && out, "null argument");
        require(sdf->data && sdf->nx >= 2 && sdf->ny >= 2 && sdf->nz >= 2, "SDF needs >= 2 nodes per axis");
        require(sdf->dx > 0 && sim_dx > 0, "dx must be positive");
        *out = nullptr;
        check_device();
        int dev = options ? options->device : -1;
        DeviceScope ds(dev);
        sdr_solver* s = new sdr_solver();
        try {
            CK(cudaGetDevice(&s->device));
            cudaDeviceProp prop;
            CK(cudaGetDeviceProperties(&prop, s->device));
            if (prop.major != 10)
                throw Fail{SDR_ERR_NO_DEVICE, "this library is built for sm_100a (B200); device is sm_" +
                                                  std::to_string(prop.major) + std::to_string(prop.minor)};
            if (g_engine_stream) {
                s->st = g_engine_stream;
                s->own_stream = false;
            } else {
                CK(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
            }
            s->create_events();
            s->shared_gpu = options && (options->flags & SDR_SOLVER_SHARED_GPU);
            if (options && (options->flags & SDR_SOLVER_BLOCKING_SYNC))
                CK(cudaEventCreateWithFlags(&s->ev_block, cudaEventBlockingSync | cudaEventDisableTiming));
            CK(cudaFuncSetAttribute(k_pcg, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPcgSmem));
            CK(cudaFuncSetAttribute(k_redist_replay, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRedistSmem));
            s->fluid = *fluid;
            s->needle = *needle;
            s->snx = (int)sdf->nx; s->sny = (int)sdf->ny; s->snz = (int)sdf->nz;
            s->sdx = sdf->dx;
            s->sox = sdf->origin.x; s->soy = sdf->origin.y; s->soz = sdf->origin.z;
            // Solver::new grid (solver.rs:185-190)
            double bx = s->sox + (double)(s->snx - 1) * s->sdx, by = s->soy + (double)(s->sny - 1) * s->sdx,
                   bz = s->soz + (double)(s->snz - 1) * s->sdx;
            double sx = bx - s->sox, sy = by - s->soy, sz = bz - s->soz;
            size_t nx = (size_t)std::fmax(std::ceil(sx / sim_dx), 1.0);
            size_t ny = (size_t)std::fmax(std::ceil(sy / sim_dx), 1.0);
            size_t nz = (size_t)std::fmax(std::ceil(sz / sim_dx), 1.0);
            require(nx * ny * nz < (size_t)INT32_MAX / 8, "grid too large");
            require(nx >= 2 && ny >= 2 && nz >= 2, "grid needs >= 2 cells per axis");
            Grid& g = s->g;
            g.nx = (int)nx; g.ny = (int)ny; g.nz = (int)nz;
            g.dx = sim_dx; g.ox = s->sox; g.oy = s->soy; g.oz = s->soz;
            g.dxf = (float)sim_dx; g.oxf = (float)g.ox; g.oyf = (float)g.oy; g.ozf = (float)g.oz;
            s->ncell = nx * ny * nz;
            s->nu = (nx + 1) * ny * nz;
            s->nv = nx * (ny + 1) * nz;
            s->nw = nx * ny * (nz + 1);
            size_t sn = sdf->nx * sdf->ny * sdf->nz;
            dalloc(s->sdf64, sn, s->st);
            dalloc(s->sdf32, sn, s->st);
            CK(cudaMemcpyAsync(s->sdf64, sdf->data, sn * 8, cudaMemcpyHostToDevice, s->st));
            LAUNCH(k_f64_to_f32, blocks(sn, 256), 256, 0, s->st, s->sdf64, s->sdf32, sn);
            dalloc(s->dst, 1, s->st);
            CK(cudaMemsetAsync(s->dst, 0, sizeof(DevStatus), s->st));
            dalloc(s->rds, 1, s->st);
            CK(cudaMemsetAsync(s->rds, 0, sizeof(RedistState), s->st));
            hget(s->hst, 1);
            hget(s->h_mout, 1);
            std::memset(s->hst, 0, sizeof(DevStatus));
            s->alloc_grid();
            LAUNCH(k_cavity_and_base, blocks(s->ncell, 256), 256, 0, s->st, g, s->sdf_d(), 0, Aabb{}, s->cavity,
                   s->base, 1);
            size_t want = options && options->max_particles ? options->max_particles
                                                             : std::min<size_t>(s->ncell * 2, 1 << 22);
            s->ensure_capacity(std::max<size_t>(want, 256));
            CK(cudaStreamSynchronize(s->st));
        } catch (...) {
            s->free_all();
            delete s;
            throw;
        }
        *out = s;
    });
}

int sdr_solver_destroy(sdr_solver* s) {
    return guard([&] {
        if (!s) return;
        DeviceScope ds(s->device);
        if (s->st) cudaStreamSynchronize(s->st);
        while (!s->collectors.empty()) s->collectors.back()->release();
        s->free_all();
        delete s;
    });
}

int sdr_solver_set_outlet(sdr_solver* s, const sdr_aabb* o) {
    return guard([&] {
        require(s, "null solver");
        DeviceScope ds(s->device);
        s->has_outlet = o != nullptr;
        if (o) s->outlet = Aabb{{o->min.x, o->min.y, o->min.z}, {o->max.x, o->max.y, o->max.z}};
        s->refresh_base();
        CK(cudaStreamSynchronize(s->st));
    });
}

int sdr_solver_set_solve_params(sdr_solver* s, const sdr_solve_params* p) {
    return guard([&] {
        require(s && p, "null argument");
        s->max_iters = p->max_iters;
        s->tol = p->tol;
    });
}

int sdr_solver_set_needle(sdr_solver* s, const sdr_needle* nd) {
    return guard([&] {
        require(s && nd, "null argument");
        s->needle = *nd;
    });
}

int sdr_solver_step(sdr_solver* s, double dt) {
    return guard([&] {
        require(s, "null solver");
        require(std::isfinite(dt) && dt >= 0.0, "dt must be finite and non-negative");
        DeviceScope ds(s->device);
        s->step(dt);
    });
}

int sdr_solver_substep(sdr_solver* s, double dt) {
    return guard([&] {
        require(s, "null solver");
        require(std::isfinite(dt) && dt > 0.0, "dt must be finite and positive");
        DeviceScope ds(s->device);
        s->substep(dt);
    });
}

int sdr_solver_run_phase(sdr_solver* s, int phase, double dt) {
    return guard([&] {
        require(s, "null solver");
        DeviceScope ds(s->device);
        s->run_phase(phase, dt);
    });
}

int sdr_solver_get_stats(const sdr_solver* s, sdr_solver_stats* o) {
    return guard([&] {
        require(s && o, "null argument");
        o->time = s->time;
        o->steps = s->steps;
        o->last_pcg_iters = s->last_pcg_iters;
        o->last_substeps = s->last_substeps;
        o->particles = s->n;
        o->drained = s->drained;
        o->last_residual = s->last_residual;
        o->emit_accum = s->emit_accum;
        o->rng_state = s->rng;
        o->emitted = s->emitted;
        o->culled = s->culled;
        o->redistributed = s->redistributed;
        o->nx = s->g.nx; o->ny = s->g.ny; o->nz = s->g.nz;
        o->dx = s->g.dx;
        o->origin = sdr_vec3{s->g.ox, s->g.oy, s->g.oz};
        o->particle_substeps = s->particle_substeps;
        o->device_ms = s->device_ms;
        o->substeps_total = s->substeps_total;
    });
}

int sdr_solver_cfl(const sdr_solver* s, double* dt, double* grid_speed) {
    return guard([&] {
        require(s && (dt || grid_speed), "null argument");
        if (dt) *dt = s->cfl_dt();
        if (grid_speed) *grid_speed = s->grid_speed;
    });
}

int sdr_solver_set_candidate_capacity(sdr_solver* s, uint64_t candidates) {
    return guard([&] {
        require(s, "null solver");
        require(candidates < (uint64_t)UINT32_MAX, "candidate capacity must be below 2^32");
        DeviceScope ds(s->device);
        s->cand_limit = (size_t)candidates;
        s->cand_n = s->cand_limit ? std::min(s->cap, s->cand_limit) : s->cap;
        dalloc(s->cand, s->cand_n, s->st);
        dalloc(s->rpend, 2 * s->cand_n, s->st);
        CK(cudaStreamSynchronize(s->st));
    });
}

int sdr_debug_inject(int fault) {
    return guard([&] {
        require(fault == 0 || fault == SDR_FAULT_SDF_STAGING, "unknown fault");
        g_fault = fault;
    });
}

int sdr_solver_set_dot_order(sdr_solver* s, int reference_order) {
    return guard([&] {
        require(s, "null solver");
        s->exact_dots = reference_order != 0;
    });
}

int sdr_solver_set_pcg_ctas(sdr_solver* s, int ctas) {
    return guard([&] {
        require(s, "null solver");
        require(ctas >= 0 && ctas <= kMaxCtas, "CTAs must be 0 (automatic) or 1..16");
        s->pcg_ctas = ctas;
    });
}

int sdr_solver_set_pcg_kernel(sdr_solver* s, int kernel) {
    return guard([&] {
        require(s, "null solver");
        if (kernel != SDR_PCG_AUTO && kernel != SDR_PCG_ONE_BLOCK && kernel != SDR_PCG_CLUSTER && kernel != SDR_PCG_TILES)
            throw Fail{SDR_ERR_INVALID, "unknown pressure-solve kernel " + std::to_string(kernel)};
        s->pcg_kernel = kernel;
    });
}

int sdr_solver_set_profiling(sdr_solver* s, int on) {
    return guard([&] {
        require(s, "null solver");
        s->profiling = on != 0;
        s->kernel_timers = on >= 2;
    });
}

int sdr_solver_get_profile(const sdr_solver* s, sdr_profile* out) {
    return guard([&] {
        require(s && out, "null argument");
        *out = s->prof;
    });
}

int sdr_solver_reset_profile(sdr_solver* s) {
    return guard([&] {
        require(s, "null solver");
        DeviceScope ds(s->device);
        s->prof = sdr_profile{};
        CK(cudaMemsetAsync(s->dst->pcg_cycles, 0, sizeof(s->dst->pcg_cycles), s->st));
        CK(cudaStreamSynchronize(s->st));
    });
}

int sdr_solver_set_scalars(sdr_solver* s, double time, double emit_accum, uint64_t steps, uint64_t drained,
                           uint64_t rng_state) {
    return guard([&] {
        require(s, "null solver");
        DeviceScope ds(s->device);
        s->time = time;
        s->emit_accum = emit_accum;
        s->steps = steps;
        s->rng = rng_state;
        s->drained = drained;
        unsigned long long d = drained;
        CK(cudaMemcpyAsync(&s->dst->drained, &d, sizeof(d), cudaMemcpyHostToDevice, s->st));
        CK(cudaStreamSynchronize(s->st));
    });
}

int sdr_solver_copy_particles(sdr_solver* s, double* pos_xyz, double* vel_xyz, size_t cap, size_t* n_out) {
    return guard([&] {
        require(s, "null solver");
        if (n_out) *n_out = s->n;
        if (cap < s->n) throw Fail{SDR_ERR_BUFFER, "buffer smaller than the particle count"};
        DeviceScope ds(s->device);
        std::vector<float4> tmp(s->n);
        for (int which = 0; which < 2; ++which) {
            double* dstp = which == 0 ? pos_xyz : vel_xyz;
            if (!dstp || !s->n) continue;
            CK(cudaMemcpyAsync(tmp.data(), which == 0 ? s->pos : s->vel, s->n * sizeof(float4),
                               cudaMemcpyDeviceToHost, s->st));
            CK(cudaStreamSynchronize(s->st));
            for (size_t i = 0; i < s->n; ++i) {
                dstp[3 * i] = tmp[i].x;
                dstp[3 * i + 1] = tmp[i].y;
                dstp[3 * i + 2] = tmp[i].z;
            }
        }
    });
}

int sdr_solver_copy_particles_f32(sdr_solver* s, float* pos_xyz, float* vel_xyz, size_t cap, size_t* n_out) {
    return guard([&] {
        require(s, "null solver");
        if (n_out) *n_out = s->n;
        if (cap < s->n) throw Fail{SDR_ERR_BUFFER, "buffer smaller than the particle count"};
        DeviceScope ds(s->device);
        if (!s->n) return;
        for (int which = 0; which < 2; ++which) {
            float* dstp = which == 0 ? pos_xyz : vel_xyz;
            if (!dstp) continue;
            CK(cudaMemcpy2DAsync(dstp, 3 * sizeof(float), which == 0 ? s->pos : s->vel, sizeof(float4),
                                 3 * sizeof(float), s->n, cudaMemcpyDeviceToHost, s->st));
        }
        CK(cudaStreamSynchronize(s->st));
    });
}

int sdr_solver_set_particles(sdr_solver* s, const double* pos_xyz, const double* vel_xyz, size_t n) {
    return guard([&] {
        require(s && (n == 0 || (pos_xyz && vel_xyz)), "null argument");
        require(n < (size_t)UINT32_MAX / 2, "too many particles");
        DeviceScope ds(s->device);
        s->ensure_capacity(n);
        if (n) {
            double* tmp = nullptr;
            CK(cudaMalloc((void**)&tmp, n * 3 * sizeof(double)));
            try {
                CK(cudaMemcpyAsync(tmp, pos_xyz, n * 24, cudaMemcpyHostToDevice, s->st));
                LAUNCH(k_pack_particles, blocks(n, 256), 256, 0, s->st, tmp, s->pos, n);
                CK(cudaMemcpyAsync(tmp, vel_xyz, n * 24, cudaMemcpyHostToDevice, s->st));
                LAUNCH(k_pack_particles, blocks(n, 256), 256, 0, s->st, tmp, s->vel, n);
                CK(cudaStreamSynchronize(s->st));
            } catch (...) {
                cudaFree(tmp);
                throw;
            }
            cudaFree(tmp);
        }
        s->n = (uint32_t)n;
        LAUNCH(k_set_u32, 1, 1, 0, s->st, s->dn(), s->n);
        s->sorted_valid = false;
        CK(cudaStreamSynchronize(s->st));
    });
}

static int copy_dev(sdr_solver* s, const void* src, size_t bytes, void* out) {
    CK(cudaMemcpyAsync(out, src, bytes, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return 0;
}

int sdr_solver_copy_pressure(sdr_solver* s, double* out, size_t cap) {
    return guard([&] {
        require(s && out, "null argument");
        if (cap < s->ncell) throw Fail{SDR_ERR_BUFFER, "buffer smaller than the cell count"};
        DeviceScope ds(s->device);
        copy_dev(s, s->p_dense, s->ncell * 8, out);
    });
}

int sdr_solver_copy_cells(sdr_solver* s, uint8_t* out, size_t cap) {
    return guard([&] {
        require(s && out, "null argument");
        if (cap < s->ncell) throw Fail{SDR_ERR_BUFFER, "buffer smaller than the cell count"};
        DeviceScope ds(s->device);
        copy_dev(s, s->cells, s->ncell, out);
    });
}

int sdr_solver_copy_cavity_mask(sdr_solver* s, uint8_t* out, size_t cap) {
    return guard([&] {
        require(s && out, "null argument");
        if (cap < s->ncell) throw Fail{SDR_ERR_BUFFER, "buffer smaller than the cell count"};
        DeviceScope ds(s->device);
        copy_dev(s, s->cavity, s->ncell, out);
    });
}

static float* face_ptr(sdr_solver* s, int which, size_t& len) {
    switch (which) {
        case 0: len = s->nu; return s->u;
        case 1: len = s->nv; return s->v;
        case 2: len = s->nw; return s->w;
        case 3: len = s->nu; return s->su;
        case 4: len = s->nv; return s->sv;
        case 5: len = s->nw; return s->sw;
    }
    throw Fail{SDR_ERR_INVALID, "face index must be 0..5"};
}

int sdr_solver_copy_face(sdr_solver* s, int which, double* out, size_t cap) {
    return guard([&] {
        require(s && out, "null argument");
        size_t len = 0;
        float* f = face_ptr(s, which, len);
        if (cap < len) throw Fail{SDR_ERR_BUFFER, "buffer smaller than the face count"};
        DeviceScope ds(s->device);
        std::vector<float> tmp(len);
        copy_dev(s, f, len * 4, tmp.data());
        for (size_t i = 0; i < len; ++i) out[i] = tmp[i];
    });
}

int sdr_solver_set_face(sdr_solver* s, int which, const double* in, size_t n) {
    return guard([&] {
        require(s && in, "null argument");
        size_t len = 0;
        float* f = face_ptr(s, which, len);
        require(n == len, "face length mismatch");
        DeviceScope ds(s->device);
        std::vector<float> tmp(len);
        for (size_t i = 0; i < len; ++i) tmp[i] = (float)in[i];
        CK(cudaMemcpyAsync(f, tmp.data(), len * 4, cudaMemcpyHostToDevice, s->st));
        CK(cudaStreamSynchronize(s->st));
    });
}

int sdr_solver_copy_sort(sdr_solver* s, uint32_t* keys, uint32_t* perm, size_t cap, size_t* n_out) {
    return guard([&] {
        require(s, "null solver");
        if (n_out) *n_out = s->n;
        if (cap < s->n) throw Fail{SDR_ERR_BUFFER, "buffer smaller than the particle count"};
        require(s->sorted_valid, "no counting sort for the current particle set (run the P2G phase)");
        DeviceScope ds(s->device);
        if (keys && s->n) copy_dev(s, s->key_sort, s->n * 4, keys);
        if (perm && s->n) copy_dev(s, s->perm, s->n * 4, perm);
    });
}

int sdr_solver_max_pressure(sdr_solver* s, double* out) {
    return guard([&] {
        require(s && out, "null argument");
        DeviceScope ds(s->device);
        std::vector<double> p(s->ncell);
        std::vector<uint8_t> c(s->ncell);
        copy_dev(s, s->p_dense, s->ncell * 8, p.data());
        copy_dev(s, s->cells, s->ncell, c.data());
        double m = 0.0;
        for (size_t i = 0; i < s->ncell; ++i)
            if (c[i] == FLUID) m = std::fmax(m, p[i]);
        *out = m;
    });
}

int sdr_solver_mean_pressure(sdr_solver* s, double* out) {
    return guard([&] {
        require(s && out, "null argument");
        DeviceScope ds(s->device);
        std::vector<double> p(s->ncell);
        std::vector<uint8_t> c(s->ncell);
        copy_dev(s, s->p_dense, s->ncell * 8, p.data());
        copy_dev(s, s->cells, s->ncell, c.data());
        double sum = 0.0;
        uint64_t k = 0;
        for (size_t i = 0; i < s->ncell; ++i)
            if (c[i] == FLUID) {
                sum += p[i];
                ++k;
            }
        *out = k ? sum / (double)k : 0.0;
    });
}

int sdr_solver_max_speed(sdr_solver* s, double* out) {
    return guard([&] {
        require(s && out, "null argument");
        DeviceScope ds(s->device);
        std::vector<float4> v(s->n);
        if (s->n) copy_dev(s, s->vel, s->n * sizeof(float4), v.data());
        double m = 0.0;
        for (auto& x : v) m = std::fmax(m, std::sqrt((double)x.x * x.x + (double)x.y * x.y + (double)x.z * x.z));
        *out = m;
    });
}

int sdr_solver_cells_fluid_count(sdr_solver* s, uint64_t* out) {
    return guard([&] {
        require(s && out, "null argument");
        DeviceScope ds(s->device);
        CK(cudaMemsetAsync(&s->dst->fluid_count, 0, 8, s->st));
        LAUNCH(k_count_fluid, blocks(s->ncell, kMetBS), kMetBS, 0, s->st, s->cells, s->ncell, &s->dst->fluid_count);
        unsigned long long v = 0;
        copy_dev(s, &s->dst->fluid_count, 8, &v);
        *out = v;
    });
}

int sdr_solver_max_particles_per_cell(sdr_solver* s, uint64_t* out) {
    return guard([&] {
        require(s && out, "null argument");
        DeviceScope ds(s->device);
        s->classify(false);
        CK(cudaMemsetAsync(&s->dst->hist_max, 0, 4, s->st));
        LAUNCH(k_hist_max, 148, 256, 0, s->st, s->hist_valid, s->ncell, &s->dst->hist_max);
        uint32_t v = 0;
        copy_dev(s, &s->dst->hist_max, 4, &v);
        *out = v;
    });
}

// ---------------------------------------------------------------- metrics
int sdr_metrics_create(sdr_solver* s, double cavity_volume, sdr_metrics** out) {
    return guard([&] {
        require(s && out, "null argument");
        DeviceScope ds(s->device);
        sdr_metrics* m = new sdr_metrics();
        try {
            m->owner = s;
            s->collectors.push_back(m);
            m->cavity_volume = cavity_volume;
            dalloc(m->is_wall, s->ncell, s->st);
            dalloc(m->washed, s->ncell, s->st);
            dalloc(m->wet, s->ncell, s->st);
            CK(cudaMemsetAsync(m->washed, 0, s->ncell, s->st));
            CK(cudaMemsetAsync(m->wet, 0, s->ncell, s->st));
            CK(cudaMemsetAsync(&s->dst->wall_count, 0, 8, s->st));
            LAUNCH(k_wall_mask, blocks(s->ncell, kMetBS), kMetBS, 0, s->st, s->g, s->cavity, m->is_wall,
                   &s->dst->wall_count);
            unsigned long long wc = 0;
            copy_dev(s, &s->dst->wall_count, 8, &wc);
            m->wall_count = wc;
        } catch (...) {
            m->release();
            delete m;
            throw;
        }
        *out = m;
    });
}

int sdr_render_slice(sdr_solver* s, const sdr_slice_plane* plane, uint32_t target_px, double vmax, uint8_t* rgb,
                     size_t cap, uint32_t* w_out, uint32_t* h_out) {
    return guard([&] {
        require(s && plane && w_out && h_out, "null argument");
        const sdr_slice_plane& p = *plane;
        require(p.hax >= 0 && p.hax < 3 && p.vax >= 0 && p.vax < 3 && p.oax >= 0 && p.oax < 3 && p.hax != p.vax &&
                    p.hax != p.oax && p.vax != p.oax,
                "slice plane axes must be a permutation of 0, 1, 2");
        DeviceScope ds(s->device);
        // image size (render.rs:139-156) from the solid SDF's bounds
        RenderView v{};
        v.hax = p.hax; v.vax = p.vax; v.oax = p.oax;
        v.flip_v = p.flip_v ? 1 : 0; v.project = p.project ? 1 : 0; v.amber = p.amber ? 1 : 0;
        v.slice = p.slice; v.slab = p.slab;
        const double org[3] = {s->sox, s->soy, s->soz};
        const int nn[3] = {s->snx, s->sny, s->snz};
        for (int a = 0; a < 3; ++a) {
            v.mn[a] = org[a];
            v.mx[a] = org[a] + (double)(nn[a] - 1) * s->sdx;
        }
        v.wm = std::fmax(v.mx[v.hax] - v.mn[v.hax], 1e-9);
        v.hm = std::fmax(v.mx[v.vax] - v.mn[v.vax], 1e-9);
        const uint32_t t = target_px > 1 ? target_px : 1;
        if (v.wm >= v.hm) {
            v.w = t;
            v.h = (uint32_t)std::fmax(std::round((double)target_px * v.hm / v.wm), 1.0);
        } else {
            v.w = (uint32_t)std::fmax(std::round((double)target_px * v.wm / v.hm), 1.0);
            v.h = t;
        }
        *w_out = v.w;
        *h_out = v.h;
        const size_t npx = (size_t)v.w * v.h;
        if (!rgb || cap < 3 * npx)
            throw Fail{SDR_ERR_BUFFER, "image buffer too small: need " + std::to_string(3 * npx) + " bytes"};
        cudaStream_t st = s->st;
        uint8_t* img = nullptr;
        dalloc(img, 3 * npx, st);
        LAUNCH(k_render_bg, blocks(npx, 256), 256, 0, st, v, s->sdf_d(), img);
        const uint32_t n = s->n;
        uint32_t *owner = nullptr, *key = nullptr, *hist = nullptr, *start = nullptr, *fill = nullptr,
                 *perm = nullptr, *longl = nullptr, *tmp = nullptr, *lcount = nullptr;
        unsigned long long* peak = nullptr;
        int2* cxy = nullptr;
        if (v.amber) {  // draw_amber_pool (render.rs:238-308)
            const double longest = (double)std::max(v.w, v.h);
            const int r = (int)std::fmax(std::round(longest / 80.0), 3.0);
            const int T = r;
            const int ntx = (int)((v.w + T - 1) / T), nty = (int)((v.h + T - 1) / T);
            const uint32_t nb = (uint32_t)(ntx + 2) * (uint32_t)(nty + 2) + 1;  // with the dump bin
            dalloc(hist, nb + 1, st);
            dalloc(start, nb + 1, st);
            dalloc(fill, nb, st);
            dalloc(longl, nb, st);
            dalloc(lcount, 1, st);
            dalloc(key, n, st);
            dalloc(cxy, n, st);
            dalloc(perm, n, st);
            dalloc(tmp, n, st);
            CK(cudaMemsetAsync(hist, 0, (nb + 1) * 4, st));
            CK(cudaMemsetAsync(lcount, 0, 4, st));
            if (n) LAUNCH(k_render_amber_keys, blocks(n, 256), 256, 0, st, v, s->pos, n, T, ntx, nty, key, cxy, hist);
            s->scan(hist, start, nb + 1, nullptr, __LINE__);
            CK(cudaMemcpyAsync(fill, start, nb * 4, cudaMemcpyDeviceToDevice, st));
            if (n) LAUNCH(k_sort_scatter, blocks(n, 256), 256, 0, st, key, n, fill, perm);
            LAUNCH(k_sort_segments, blocks(nb, 256), 256, 0, st, start, nb, perm, longl, lcount);
            LAUNCH(k_sort_long, 148, 256, 0, st, start, longl, lcount, perm, tmp);
            LAUNCH(k_render_amber_pixels, blocks(npx, 256), 256, 0, st, v, r, T, ntx, start, perm, cxy, img);
        } else {  // speed-coloured dots (render.rs:201-221)
            dalloc(owner, npx, st);
            dalloc(peak, 1, st);
            CK(cudaMemsetAsync(owner, 0, npx * 4, st));
            CK(cudaMemsetAsync(peak, 0, 8, st));
            if (n && !(vmax > 0.0)) LAUNCH(k_render_max_speed, blocks(n, 256), 256, 0, st, s->vel, n, peak);
            if (n) LAUNCH(k_render_dots_mark, blocks(n, 256), 256, 0, st, v, s->pos, n, owner);
            LAUNCH(k_render_dots_color, blocks(npx, 256), 256, 0, st, v, s->vel, owner, peak, vmax, img);
        }
        copy_dev(s, img, 3 * npx, rgb);
        for (auto* q : {owner, key, hist, start, fill, perm, longl, tmp, lcount}) {
            uint32_t* qq = q;
            dfree(qq, st);
        }
        dfree(peak, st);
        dfree(cxy, st);
        dfree(img, st);
        // the needle on top (render.rs:224-231): a 12 mm segment behind the tip and a disk at it
        auto to_px = [&](double x, double y, double z, int64_t& cx, int64_t& cy) {
            const double a[3] = {x, y, z};
            const double fx = (a[v.hax] - v.mn[v.hax]) / v.wm * (double)v.w;
            const double fy = v.flip_v ? (v.mx[v.vax] - a[v.vax]) / v.hm * (double)v.h
                                       : (a[v.vax] - v.mn[v.vax]) / v.hm * (double)v.h;
            auto cvt = [](double f) -> int64_t {
                if (std::isnan(f)) return 0;
                if (f >= 9223372036854775807.0) return INT64_MAX;
                if (f <= -9223372036854775808.0) return INT64_MIN;
                return (int64_t)f;
            };
            cx = cvt(fx);
            cy = cvt(fy);
        };
        const sdr_vec3 tip = s->needle.tip, ax = s->needle.axis;
        int64_t bx0, by0, tx0, ty0;
        to_px(tip.x - ax.x * 0.012, tip.y - ax.y * 0.012, tip.z - ax.z * 0.012, bx0, by0);
        to_px(tip.x, tip.y, tip.z, tx0, ty0);
        const uint8_t needle[3] = {255, 80, 80};
        sdr_internal_draw_line(rgb, v.w, v.h, bx0, by0, tx0, ty0, needle);
        sdr_internal_draw_disk(rgb, v.w, v.h, tx0, ty0, 3, needle);
    });
}

int sdr_metrics_write_json(const sdr_metrics* m, const char* path) {
    return guard([&] {
        require(m && path, "null argument");
        std::string err;
        int rc = sdr_internal_write_text(path, sdr_internal_frames_json(m->history.data(), m->history.size()), err);
        if (rc != SDR_OK) throw Fail{rc, err};
    });
}

int sdr_metrics_write_csv(const sdr_metrics* m, const char* path) {
    return guard([&] {
        require(m && path, "null argument");
        std::string err;
        int rc = sdr_internal_write_text(path, sdr_internal_frames_csv(m->history.data(), m->history.size()), err);
        if (rc != SDR_OK) throw Fail{rc, err};
    });
}

int sdr_metrics_destroy(sdr_metrics* m) {
    return guard([&] {
        if (!m) return;
        if (m->owner) {
            DeviceScope ds(m->owner->device);
            m->release();
        }
        delete m;
    });
}

int sdr_metrics_record(sdr_metrics* m, sdr_solver* s, uint64_t frame, sdr_frame_metrics* out) {
    return guard([&] {
        require(m && s, "null argument");
        require(m->owner == s, "metrics collector belongs to another solver");
        DeviceScope ds(s->device);
        const double M3_TO_ML = 1.0e6, PA_TO_MMHG = 1.0 / 133.322, CAP_FACTOR = 3.0;
        unsigned npb = blocks(std::max<uint32_t>(s->n, 1), kMetBS);
        if (npb * 2 > s->mpart_cap) {
            dalloc(s->mpart, (size_t)npb * 2);
            s->mpart_cap = (size_t)npb * 2;
        }
        if (s->n)
            LAUNCH(k_metrics_particles, npb, kMetBS, 0, s->st, s->g, s->pos, s->vel, s->n, m->is_wall, m->washed,
                   m->wet, s->mpart);
        else
            npb = 0;
        double v_jet = s->jet_speed();
        double stagnation = 0.5 * s->fluid.density * v_jet * v_jet;
        double gl = std::sqrt(s->fluid.gravity.x * s->fluid.gravity.x + s->fluid.gravity.y * s->fluid.gravity.y +
                              s->fluid.gravity.z * s->fluid.gravity.z);
        double hydrostatic = s->fluid.density * gl * ((double)s->g.ny * s->g.dx);
        double p_cap = CAP_FACTOR * stagnation + hydrostatic + 500.0;  // metrics.rs:232-236
        unsigned ncb = blocks(s->ncell, kMetBS);
        LAUNCH(k_metrics_cells, ncb, kMetBS, 0, s->st, s->ncell, s->cells, s->p_dense, m->washed, m->wet, p_cap,
               s->mcell);
        LAUNCH(k_metrics_final, 1, 32, 0, s->st, s->mcell, (int)ncb, s->mpart, (int)npb, s->mout);
        copy_dev(s, s->mout, sizeof(MetricsOut), s->h_mout);
        const MetricsOut& o = *s->h_mout;
        double pv = s->particle_volume();
        double fluid_volume = (double)s->n * pv;
        double drained_volume = (double)s->drained * pv;
        double fill = m->cavity_volume > 0.0 ? fluid_volume / m->cavity_volume : 0.0;
        m->injected_ml = (fluid_volume + drained_volume) * M3_TO_ML;
        sdr_frame_metrics f{};
        f.frame = frame;
        f.time_s = s->time;
        f.particles = s->n;
        f.fluid_volume_ml = fluid_volume * M3_TO_ML;
        f.drained_volume_ml = drained_volume * M3_TO_ML;
        f.fill_fraction = fill;
        f.wall_coverage = m->wall_count > 0 ? (double)o.washed / (double)m->wall_count : 0.0;
        f.mean_pressure_pa = o.fl_n ? o.fl_sum / (double)o.fl_n : 0.0;
        f.max_pressure_pa = o.fl_max;
        f.max_pressure_mmhg = o.fl_max * PA_TO_MMHG;
        f.wall_pressure_pa = o.ww_n ? o.ww_sum / (double)o.ww_n : 0.0;
        f.peak_wall_pressure_pa = o.ww_n ? o.ww_peak : 0.0;
        f.peak_wall_pressure_mmhg = f.peak_wall_pressure_pa * PA_TO_MMHG;
        f.membrane_artifacts = o.ww_art;
        f.max_speed_m_s = o.max_speed;
        f.kinetic_energy = 0.5 * o.ke_sum;
        f.pcg_iters = s->last_pcg_iters;
        m->history.push_back(f);
        if (out) *out = f;
    });
}

int sdr_metrics_summary(const sdr_metrics* m, sdr_summary* out) {  // metrics.rs:324-382
    return guard([&] {
        require(m && out, "null argument");
        const double PA_TO_MMHG = 1.0 / 133.322;
        double peak_fill = 0, peak_cov = 0, peak_p = 0, peak_mem = 0, mean_mem = 0;
        uint64_t art = 0;
        for (auto& f : m->history) {
            peak_fill = std::fmax(peak_fill, f.fill_fraction);
            peak_cov = std::fmax(peak_cov, f.wall_coverage);
            peak_p = std::fmax(peak_p, f.max_pressure_pa);
            peak_mem = std::fmax(peak_mem, f.peak_wall_pressure_pa);
            art += f.membrane_artifacts;
        }
        if (!m->history.empty()) {
            double sum = -0.0;
            for (auto& f : m->history) sum += f.wall_pressure_pa;
            mean_mem = sum / (double)m->history.size();
        }
        const sdr_frame_metrics* last = m->history.empty() ? nullptr : &m->history.back();
        sdr_summary s{};
        s.frames = m->history.size();
        s.final_time_s = last ? last->time_s : 0.0;
        s.peak_fill_fraction = peak_fill;
        s.final_fill_fraction = last ? last->fill_fraction : 0.0;
        s.peak_wall_coverage = peak_cov;
        s.final_wall_coverage = last ? last->wall_coverage : 0.0;
        s.peak_membrane_pressure_pa = peak_mem;
        s.peak_membrane_pressure_mmhg = peak_mem * PA_TO_MMHG;
        s.mean_membrane_pressure_pa = mean_mem;
        s.mean_membrane_pressure_mmhg = mean_mem * PA_TO_MMHG;
        s.peak_pressure_pa = peak_p;
        s.peak_pressure_mmhg = peak_p * PA_TO_MMHG;
        s.membrane_artifacts_total = art;
        double resident = last ? last->fluid_volume_ml : 0.0, drained = last ? last->drained_volume_ml : 0.0;
        s.total_drained_ml = drained;
        s.injected_ml = resident + drained;
        s.mass_balance = m->injected_ml > 0.0 ? s.injected_ml / m->injected_ml : 1.0;
        *out = s;
    });
}

int sdr_metrics_wall_count(const sdr_metrics* m, uint64_t* out) {
    return guard([&] {
        require(m && out, "null argument");
        *out = m->wall_count;
    });
}

// ---------------------------------------------------------------- geometry
int sdr_sdf_mesh_grid(const double* tris, size_t ntri, double dx, double padding, sdr_vec3* origin,
                      uint64_t dims[3]) {
    return guard([&] {
        require(tris && ntri && origin && dims && dx > 0, "bad argument");
        double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (size_t v = 0; v < 3 * ntri; ++v)
            for (int c = 0; c < 3; ++c) {
                mn[c] = std::fmin(mn[c], tris[3 * v + c]);
                mx[c] = std::fmax(mx[c], tris[3 * v + c]);
            }
        for (int c = 0; c < 3; ++c) {
            mn[c] -= padding;
            mx[c] += padding;
            dims[c] = (uint64_t)std::ceil((mx[c] - mn[c]) / dx) + 1;
        }
        *origin = sdr_vec3{mn[0], mn[1], mn[2]};
    });
}

int sdr_sdf_from_mesh(const double* tris, size_t ntri, sdr_vec3 origin, double dx, const uint64_t dims[3],
                      double* out) {
    return guard([&] {
        require(tris && ntri && dims && out && dx > 0, "bad argument");
        const size_t nn = sdf_node_count(dims);
        require(ntri <= (size_t)UINT32_MAX / 2, "too many triangles");
        check_device();
        const uint32_t skip = g_fault == SDR_FAULT_SDF_STAGING ? 0u : kNoSkip;
        g_fault = 0;
        uint32_t ntiles = (uint32_t)((ntri + kSdfTile - 1) / kSdfTile);
        size_t padded = (size_t)ntiles * kSdfTile * 9;
        double *dt = nullptr, *dout = nullptr;
        uint32_t* derr = nullptr;
        cudaStream_t st = nullptr;
        auto cleanup = [&] {
            if (dt) cudaFree(dt);
            if (dout) cudaFree(dout);
            if (derr) cudaFree(derr);
            if (st) cudaStreamDestroy(st);
        };
        try {
            CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            CK(cudaMalloc((void**)&dt, padded * 8));
            CK(cudaMalloc((void**)&dout, nn * 8));
            CK(cudaMalloc((void**)&derr, 4));
            CK(cudaMemsetAsync(dt, 0, padded * 8, st));
            CK(cudaMemsetAsync(derr, 0, 4, st));
            CK(cudaMemcpyAsync(dt, tris, ntri * 72, cudaMemcpyHostToDevice, st));
            LAUNCH(k_sdf_mesh, blocks(nn, kSdfBS), kSdfBS, 0, st, dt, (uint32_t)ntri, ntiles, origin.x, origin.y,
                   origin.z, dx, (int)dims[0], (int)dims[1], (int)dims[2], dout, derr, skip);
            CK(cudaMemcpyAsync(out, dout, nn * 8, cudaMemcpyDeviceToHost, st));
            uint32_t e = 0;
            CK(cudaMemcpyAsync(&e, derr, 4, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (e) throw Fail{SDR_ERR_DEVICE_TIMEOUT, "triangle staging wait gave up"};
        } catch (...) {
            cleanup();
            throw;
        }
        cleanup();
    });
}

int sdr_sdf_from_mesh_noalloc(const double* tris_dev, size_t ntri, sdr_vec3 origin, double dx,
                              const uint64_t dims[3], double* out_dev, void* stream) {
    return guard([&] {
        require(tris_dev && out_dev && dims && ntri && dx > 0, "bad argument");
        if (ntri > (size_t)SDR_NOALLOC_MAX_TRIANGLES)
            throw Fail{SDR_ERR_INVALID, "mesh has " + std::to_string(ntri) + " triangles; the no-allocation scratch holds " +
                                            std::to_string(SDR_NOALLOC_MAX_TRIANGLES)};
        require(((uintptr_t)out_dev & 7) == 0, "out_dev must be 8-byte aligned");
        const size_t nn = sdf_node_count(dims);
        check_device();
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        double* tiles = noalloc_scratch();
        uint32_t* err = reinterpret_cast<uint32_t*>(tiles + kNoAllocTris * 9);
        uint32_t ntiles = (uint32_t)((ntri + kSdfTile - 1) / kSdfTile);
        size_t used = ntri * 9, padded = (size_t)ntiles * kSdfTile * 9;
        // The scratch keeps the previous call's contents: overwrite the
        // triangles, zero the padding tail and the error word.
        CK(cudaMemcpyAsync(tiles, tris_dev, used * sizeof(double), cudaMemcpyDeviceToDevice, st));
        if (padded > used) CK(cudaMemsetAsync(tiles + used, 0, (padded - used) * sizeof(double), st));
        CK(cudaMemsetAsync(err, 0, sizeof(uint32_t), st));
        LAUNCH(k_sdf_mesh, blocks(nn, kSdfBS), kSdfBS, 0, st, tiles, (uint32_t)ntri, ntiles, origin.x, origin.y,
               origin.z, dx, (int)dims[0], (int)dims[1], (int)dims[2], out_dev, err);
        uint32_t e = 0;
        CK(cudaMemcpyAsync(&e, err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (e) throw Fail{SDR_ERR_DEVICE_TIMEOUT, "triangle staging wait gave up"};
    });
}

int sdr_sdf_from_sinus(const sdr_sinus_params* p, sdr_vec3 origin, double dx, const uint64_t dims[3],
                       double* out) {
    return guard([&] {
        require(p && dims && out && dx > 0, "bad argument");
        const size_t nn = sdf_node_count(dims);
        check_device();
        double* dout = nullptr;
        cudaStream_t st = nullptr;
        try {
            CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            CK(cudaMalloc((void**)&dout, nn * 8));
            SinusD sd{p->semi_axes.x, p->semi_axes.y, p->semi_axes.z, p->center.x, p->center.y, p->center.z,
                      p->taper, p->bumpiness, p->socket_x, p->socket_z, p->socket_radius, p->socket_depth};
            LAUNCH(k_sdf_sinus, blocks(nn, 256), 256, 0, st, sd, origin.x, origin.y, origin.z, dx, (int)dims[0],
                   (int)dims[1], (int)dims[2], dout);
            CK(cudaMemcpyAsync(out, dout, nn * 8, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
        } catch (...) {
            if (dout) cudaFree(dout);
            if (st) cudaStreamDestroy(st);
            throw;
        }
        cudaFree(dout);
        cudaStreamDestroy(st);
    });
}

}  // extern "C"

// ================================================================= frame writer
// Double-buffered per-frame particle output (see sdr_frame_writer_* in the
// header): the D2H copy is queued on the solver's stream, the file is written
// by a thread once the copy's event fires.
int sdr_internal_write_points(const char* path, int32_t format, const float* xyz, size_t stride, size_t n,
                              std::string& err);
std::string sdr_internal_frame_path(const char* dir, const char* prefix, uint64_t frame, int32_t format);

struct sdr_frame_writer {
    std::string dir, prefix;
    int32_t format = SDR_FORMAT_VTK;
    float4* host[2] = {nullptr, nullptr};  // pinned
    size_t cap[2] = {0, 0};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    int ev_device[2] = {-1, -1};
    size_t count[2] = {0, 0};
    uint64_t frame[2] = {0, 0};
    bool busy[2] = {false, false};  // submitted and not yet written
    int next = 0;
    std::deque<int> ready;
    std::mutex mu;
    std::condition_variable cv;
    std::thread th;
    bool stop = false;
    int err_code = SDR_OK;
    std::string err;

    void loop() {
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            cv.wait(lk, [&] { return stop || !ready.empty(); });
            if (ready.empty()) return;  // stopping and drained
            const int slot = ready.front();
            ready.pop_front();
            lk.unlock();
            int rc = SDR_OK;
            std::string msg;
            if (ev_device[slot] >= 0) cudaSetDevice(ev_device[slot]);
            cudaError_t e = cudaEventSynchronize(ev[slot]);
            if (e != cudaSuccess) {
                rc = SDR_ERR_CUDA;
                msg = std::string("frame copy: ") + cudaGetErrorString(e);
            } else {
                std::string path = sdr_internal_frame_path(dir.c_str(), prefix.c_str(), frame[slot], format);
                rc = sdr_internal_write_points(path.c_str(), format, reinterpret_cast<const float*>(host[slot]), 4,
                                               count[slot], msg);
            }
            lk.lock();
            if (rc != SDR_OK && err_code == SDR_OK) {
                err_code = rc;
                err = msg;
            }
            busy[slot] = false;
            cv.notify_all();
        }
    }
};

extern "C" {

int sdr_frame_writer_create(const char* dir, const char* prefix, int32_t format, sdr_frame_writer** out) {
    return guard([&] {
        require(dir && prefix && out, "null argument");
        require(format == SDR_FORMAT_VTK || format == SDR_FORMAT_XYZ, "unknown output format");
        *out = nullptr;
        auto w = std::make_unique<sdr_frame_writer>();
        w->dir = dir;
        w->prefix = prefix;
        w->format = format;
        w->th = std::thread([p = w.get()] { p->loop(); });
        *out = w.release();
    });
}

int sdr_frame_writer_submit(sdr_frame_writer* w, sdr_solver* s, uint64_t frame) {
    return guard([&] {
        require(w && s, "null argument");
        DeviceScope ds(s->device);
        std::unique_lock<std::mutex> lk(w->mu);
        if (w->err_code != SDR_OK) throw Fail{w->err_code, w->err};
        const int slot = w->next;
        w->cv.wait(lk, [&] { return !w->busy[slot]; });  // its previous file is written
        if (w->err_code != SDR_OK) throw Fail{w->err_code, w->err};
        w->busy[slot] = true;
        lk.unlock();
        try {
            const size_t n = s->n;
            if (n > w->cap[slot]) {
                if (w->host[slot]) hput(w->host[slot], w->cap[slot]);
                w->cap[slot] = 0;
                size_t c = std::max<size_t>(n + n / 2, 4096);
                hget(w->host[slot], c, &c);
                w->cap[slot] = c;
            }
            if (!w->ev[slot] || w->ev_device[slot] != s->device) {
                if (w->ev[slot]) cudaEventDestroy(w->ev[slot]);
                w->ev[slot] = nullptr;
                CK(cudaEventCreateWithFlags(&w->ev[slot], cudaEventDisableTiming));
                w->ev_device[slot] = s->device;
            }
            if (n) CK(cudaMemcpyAsync(w->host[slot], s->pos, n * sizeof(float4), cudaMemcpyDeviceToHost, s->st));
            CK(cudaEventRecord(w->ev[slot], s->st));
        } catch (...) {
            lk.lock();
            w->busy[slot] = false;
            w->cv.notify_all();
            throw;
        }
        lk.lock();
        w->count[slot] = s->n;
        w->frame[slot] = frame;
        w->ready.push_back(slot);
        w->next ^= 1;
        w->cv.notify_all();
    });
}

int sdr_frame_writer_flush(sdr_frame_writer* w) {
    return guard([&] {
        require(w, "null writer");
        std::unique_lock<std::mutex> lk(w->mu);
        w->cv.wait(lk, [&] { return !w->busy[0] && !w->busy[1]; });
        if (w->err_code != SDR_OK) throw Fail{w->err_code, w->err};
    });
}

int sdr_frame_writer_destroy(sdr_frame_writer* w) {
    if (!w) return SDR_OK;
    {
        std::lock_guard<std::mutex> lk(w->mu);
        w->stop = true;
    }
    w->cv.notify_all();
    if (w->th.joinable()) w->th.join();
    const int rc = w->err_code;
    const std::string msg = w->err;
    for (int i = 0; i < 2; ++i) {
        if (w->host[i]) hput(w->host[i], w->cap[i]);
        if (w->ev[i]) cudaEventDestroy(w->ev[i]);
    }
    delete w;
    if (rc != SDR_OK) g_err = msg;
    return rc;
}

}  // extern "C"

// ================================================================= packed batches
// Many scenes advanced together: every packed step runs one substep of every
// live scene (each at its own CFL step, Solver::step's arithmetic per scene),
// with one launch per substep operation for all of them (packed.cuh). Scenes
// join and leave between packed steps; a scene's frames, metrics and summary
// are its own.
#include "packed_engine.h"

struct PackedEngine {
    struct Scene {
        uint64_t tag = 0;
        sdr_solver* s = nullptr;
        sdr_metrics* m = nullptr;
        double frame_dt = 0, remaining = 0, floor_ = 0, sub = 0;
        uint64_t frame = 0, frames = 0;
        uint32_t taken = 0;
    };
    int device = 0;
    cudaStream_t st = nullptr;
    Packer pk;
    std::vector<Scene> live;
    unsigned grid_cap = 0;
    unsigned char* dev_arena = nullptr;
    size_t dev_cap = 0;
    unsigned char* host_arena = nullptr;  // pinned
    size_t host_cap = 0;
    uint64_t launches = 0, steps = 0, captures = 0;
    // the packed step as a CUDA graph, replayed while its launch plan is unchanged
    std::vector<PackStep> plan, graph_plan;
    const unsigned char* graph_arena = nullptr;
    cudaGraphExec_t gexec = nullptr;
    // autotuner of the persistent grid cap: candidate CTAs per SM, each timed
    // over kTuneSteps packed steps (CUDA events), then the fastest kept
    int nsm = 0;
    static constexpr int kTuneCaps[4] = {2, 4, 8, 16};
    static constexpr int kTuneSteps = 3;
    int tune = 0;                 // candidate under test (4: done)
    int tune_n = 0;               // its steps so far
    double tune_ms[4] = {0, 0, 0, 0};
    double tune_work[4] = {0, 0, 0, 0};  // particle-substeps of those steps
    int chosen = 8;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    unsigned cap() const { return (unsigned)nsm * (unsigned)(tune < 4 ? kTuneCaps[tune] : chosen); }

    // One packed step's launches: the graph captured from the same plan and
    // arena if there is one, else a new capture.
    void launch(const unsigned char* dev) {
        if (!(gexec && dev == graph_arena && plan == graph_plan)) {
            for (auto& p : plan) CK(p.prep(p.smem));
            if (gexec) cudaGraphExecDestroy(gexec);
            gexec = nullptr;
            cudaGraph_t graph = nullptr;
            CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            for (auto& p : plan) p.fn(dev + p.hdr_at, p.grid, p.threads, p.smem, st);
            const cudaError_t le = cudaGetLastError();
            CK(cudaStreamEndCapture(st, &graph));
            if (le != cudaSuccess) {
                cudaGraphDestroy(graph);
                throw Fail{SDR_ERR_CUDA, std::string("packed launch: ") + cudaGetErrorString(le)};
            }
            const cudaError_t ie = cudaGraphInstantiate(&gexec, graph, 0);
            cudaGraphDestroy(graph);
            CK(ie);
            graph_plan = plan;
            graph_arena = dev;
            captures += 1;
        }
        CK(cudaGraphLaunch(gexec, st));
        launches += plan.size();
        g_launches.fetch_add(plan.size(), std::memory_order_relaxed);
    }

    void finish(Scene& sc, int status, const std::string& err, std::vector<PackedDone>& done) {
        PackedDone d;
        d.tag = sc.tag;
        d.status = status;
        d.error = err;
        if (status == SDR_OK) {
            if (sdr_metrics_summary(sc.m, &d.summary) != SDR_OK || sdr_solver_get_stats(sc.s, &d.stats) != SDR_OK) {
                d.status = SDR_ERR_CUDA;
                d.error = sdr_last_error();
            }
        }
        if (sc.m) sdr_metrics_destroy(sc.m);
        if (sc.s) sdr_solver_destroy(sc.s);
        sc.m = nullptr;
        sc.s = nullptr;
        done.push_back(std::move(d));
    }
};

PackedEngine* packed_engine_create(int32_t device) {
    auto* e = new PackedEngine();
    try {
        check_device();
        DeviceScope ds(device);
        CK(cudaGetDevice(&e->device));
        CK(cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking));
        int nsm = 0;
        CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, e->device));
        e->nsm = nsm;
        CK(cudaEventCreate(&e->ev0));
        CK(cudaEventCreate(&e->ev1));
    } catch (const Fail& f) {
        if (e->st) cudaStreamDestroy(e->st);
        delete e;
        sdr_internal_set_error(f.msg);
        return nullptr;
    }
    return e;
}

int packed_engine_add(PackedEngine* e, const sdr_scene_desc& d, uint64_t capacity, uint64_t tag,
                      std::vector<PackedDone>& done) {
    DeviceScope ds(e->device);
    PackedEngine::Scene sc;
    sc.tag = tag;
    sdr_solver_options o{};
    o.max_particles = capacity;
    o.device = e->device;
    o.flags = SDR_SOLVER_SHARED_GPU;
    g_engine_stream = e->st;
    int rc = sdr_solver_create(&d.sdf, d.sim_dx, &d.fluid, &d.needle, &o, &sc.s);
    g_engine_stream = nullptr;
    if (rc == SDR_OK && d.has_outlet) rc = sdr_solver_set_outlet(sc.s, &d.outlet);
    if (rc == SDR_OK) rc = sdr_solver_set_solve_params(sc.s, &d.solve);
    if (rc == SDR_OK) rc = sdr_metrics_create(sc.s, d.cavity_volume, &sc.m);
    if (rc != SDR_OK) {
        e->finish(sc, rc, sdr_last_error(), done);
        return rc;
    }
    sc.frame_dt = d.frame_dt;
    sc.remaining = d.frame_dt;
    sc.floor_ = d.frame_dt / 512.0;  // solver.rs:248-249
    sc.frames = d.frames;
    if (sc.frames == 0) {
        e->finish(sc, SDR_OK, "", done);
        return SDR_OK;
    }
    e->live.push_back(sc);
    return SDR_OK;
}

size_t packed_engine_live(const PackedEngine* e) { return e->live.size(); }

void packed_engine_step(PackedEngine* e, std::vector<PackedDone>& done) {
    if (e->live.empty()) return;
    DeviceScope ds(e->device);
    std::vector<char> recorded(e->live.size(), 0);
    std::vector<std::string> errs(e->live.size());
    std::vector<int> codes(e->live.size(), SDR_OK);
    // every live scene records one substep (Solver::step's choice of dt, solver.rs:252-256)
    for (size_t q = 0; q < e->live.size(); ++q) {
        auto& sc = e->live[q];
        sc.sub = std::fmin(std::fmax(sc.s->cfl_dt(), sc.floor_), sc.remaining);
        e->pk.begin_scene();
        sc.s->pk = &e->pk;
        try {
            sc.s->substep_issue(sc.sub);
            sc.s->status_issue();
            recorded[q] = 1;
        } catch (const Fail& f) {
            e->pk.drop_scene();
            codes[q] = f.code;
            errs[q] = f.msg;
        } catch (...) {
            e->pk.drop_scene();
            codes[q] = SDR_ERR_CUDA;
            errs[q] = "substep recording failed";
        }
        sc.s->pk = nullptr;
    }
    int rc = SDR_OK;
    std::string msg;
    uint64_t work = 0;  // particle-substeps of this packed step (the autotuner's unit of work)
    for (size_t q = 0; q < e->live.size(); ++q)
        if (recorded[q]) work += e->live[q].s->pending_n_before + 1;
    try {
        const std::vector<unsigned char>& host = e->pk.build(e->cap(), e->plan);
        const size_t bytes = host.size();
        if (bytes > e->dev_cap) {
            dalloc(e->dev_arena, bytes + bytes / 2, e->st);
            e->dev_cap = bytes + bytes / 2;
        }
        if (bytes > e->host_cap) {
            CK(cudaStreamSynchronize(e->st));  // the old staging block may still be read
            if (e->host_arena) hput(e->host_arena, e->host_cap);
            e->host_cap = 0;
            hget(e->host_arena, bytes + bytes / 2, &e->host_cap);
        }
        std::memcpy(e->host_arena, host.data(), bytes);
        CK(cudaMemcpyAsync(e->dev_arena, e->host_arena, bytes, cudaMemcpyHostToDevice, e->st));
        CK(cudaEventRecord(e->ev0, e->st));
        e->launch(e->dev_arena);
        CK(cudaEventRecord(e->ev1, e->st));
        CK(cudaStreamSynchronize(e->st));
        if (e->tune < 4) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, e->ev0, e->ev1));
            if (e->tune_n > 0) {  // the first step of a candidate pays its capture
                e->tune_ms[e->tune] += ms;
                e->tune_work[e->tune] += (double)work;
            }
            if (++e->tune_n > PackedEngine::kTuneSteps) {
                e->tune_n = 0;
                if (++e->tune == 4) {
                    int best = 2;
                    double best_rate = -1.0;
                    for (int c = 0; c < 4; ++c) {
                        const double rate = e->tune_ms[c] > 0 ? e->tune_work[c] / e->tune_ms[c] : 0.0;
                        if (rate > best_rate) {
                            best_rate = rate;
                            best = c;
                        }
                    }
                    e->chosen = PackedEngine::kTuneCaps[best];
                }
            }
        }
    } catch (const Fail& f) {
        rc = f.code;
        msg = f.msg;
        cudaStreamSynchronize(e->st);
    }
    e->steps += 1;
    std::vector<PackedEngine::Scene> keep;
    for (size_t q = 0; q < e->live.size(); ++q) {
        auto& sc = e->live[q];
        if (rc != SDR_OK) {
            e->finish(sc, rc, msg, done);
            continue;
        }
        if (!recorded[q]) {
            e->finish(sc, codes[q], errs[q], done);
            continue;
        }
        try {
            sc.s->status_read();
            sc.s->substep_finish(sc.sub);
        } catch (const Fail& f) {
            e->finish(sc, f.code, f.msg, done);
            continue;
        }
        sc.remaining -= sc.sub;
        sc.taken += 1;
        if (sc.remaining > 1e-12) {
            keep.push_back(sc);
            continue;
        }
        // the frame is complete: Solver::step's bookkeeping, then MetricsCollector::record
        sc.s->last_substeps = sc.taken;
        sdr_frame_metrics fm;
        const int mrc = sdr_metrics_record(sc.m, sc.s, sc.frame, &fm);
        if (mrc != SDR_OK) {
            e->finish(sc, mrc, sdr_last_error(), done);
            continue;
        }
        sc.frame += 1;
        sc.taken = 0;
        sc.remaining = sc.frame_dt;
        if (sc.frame >= sc.frames) e->finish(sc, SDR_OK, "", done);
        else keep.push_back(sc);
    }
    e->live.swap(keep);
}

void packed_engine_counters(const PackedEngine* e, uint64_t* launches, uint64_t* steps, uint64_t* captures,
                            int* ctas_per_sm) {
    if (launches) *launches = e->launches;
    if (steps) *steps = e->steps;
    if (captures) *captures = e->captures;
    if (ctas_per_sm) *ctas_per_sm = e->tune < 4 ? 0 : e->chosen;
}

void packed_engine_destroy(PackedEngine* e) {
    if (!e) return;
    DeviceScope ds(e->device);
    std::vector<PackedDone> done;
    for (auto& sc : e->live) e->finish(sc, SDR_ERR_INVALID, "engine destroyed before the scene finished", done);
    e->live.clear();
    if (e->st) cudaStreamSynchronize(e->st);
    if (e->gexec) cudaGraphExecDestroy(e->gexec);
    if (e->ev0) cudaEventDestroy(e->ev0);
    if (e->ev1) cudaEventDestroy(e->ev1);
    dfree(e->dev_arena, e->st);
    if (e->host_arena) hput(e->host_arena, e->host_cap);
    if (e->st) {
        cudaStreamSynchronize(e->st);
        cudaStreamDestroy(e->st);
    }
    delete e;
}
