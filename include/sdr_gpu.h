/*
 * sdr_gpu.h — C ABI of the B200 (sm_100a) FLIP/PIC substep of uselessgoddess/sdr.
 *
 * This is the drop-in boundary: every entry point replaces one piece of the
 * reference's Rust API (paths are within the reference project). A Rust
 * `extern "C"` block binds these one to one.
 *
 * Conventions
 *  - Opaque handles, created and destroyed explicitly by the caller.
 *  - Every call returns an int status (SDR_OK = 0). No exceptions or longjmp
 *    cross this boundary. sdr_last_error() returns a thread-local message for
 *    the most recent failure on the calling thread.
 *  - All buffers are host memory owned by the caller; outputs are copied into
 *    them. No torch, CUDA or C++ types appear in the signatures.
 *  - One solver handle per host thread at a time; calls on one handle are not
 *    re-entrant. Each handle owns its CUDA stream on the current device.
 *  - Units are SI (metres, seconds, m^3/s), like the reference's Solver.
 */
#ifndef SDR_GPU_H
#define SDR_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SDR_ABI_VERSION 1

/* Status codes. */
enum {
    SDR_OK = 0,
    SDR_ERR_INVALID = 1,        /* bad argument (null pointer, size mismatch, bad params) */
    SDR_ERR_CUDA = 2,           /* a CUDA runtime call failed */
    SDR_ERR_OOM = 3,            /* device allocation failed */
    SDR_ERR_CAPACITY = 4,       /* particle or work-list capacity exceeded (the redistribution
                                   candidate list: see sdr_solver_set_candidate_capacity) */
    SDR_ERR_DEVICE_TIMEOUT = 5, /* a bounded device-side wait or loop gave up */
    SDR_ERR_NO_DEVICE = 6,      /* no CUDA device or the library was built for another arch */
    SDR_ERR_BUFFER = 7,         /* caller buffer too small; required size reported */
    SDR_ERR_IO = 8              /* a file could not be created or written */
};

/* Cell labels (src/pressure.rs:24-32). */
enum { SDR_CELL_SOLID = 0, SDR_CELL_FLUID = 1, SDR_CELL_AIR = 2 };

typedef struct { double x, y, z; } sdr_vec3;
typedef struct { sdr_vec3 min, max; } sdr_aabb; /* Aabb, src/math.rs:198-257 */

/* FluidParams, src/solver.rs:41-71. */
typedef struct {
    double density;
    sdr_vec3 gravity;
    double flip_ratio;
    uint64_t particles_per_cell;
    double volume_stiffness;
    int32_t redistribute;
    int32_t reserved0;
    double redist_cap_factor;
} sdr_fluid_params;

/* Needle, src/solver.rs:89-103 (inject_until = +inf injects for the whole run). */
typedef struct {
    sdr_vec3 tip;
    sdr_vec3 axis;
    double radius;
    double flow_rate;
    double inject_until;
} sdr_needle;

/* SolveParams, src/pressure.rs:36-50. */
typedef struct {
    uint64_t max_iters;
    double tol;
} sdr_solve_params;

/* A node-grid signed distance field, src/sdf.rs:23-34; data is nx*ny*nz
 * values, x fastest, phi < 0 inside the cavity. */
typedef struct {
    sdr_vec3 origin;
    double dx;
    uint64_t nx, ny, nz;
    const double* data;
} sdr_sdf_desc;

/* Optional creation settings; pass NULL for defaults. */
typedef struct {
    uint64_t max_particles; /* device particle capacity (0 = derive from the cavity volume) */
    int32_t device;         /* CUDA device ordinal (-1 = current) */
    int32_t flags;          /* SDR_SOLVER_* bits */
} sdr_solver_options;

/* The host thread sleeps while it waits for the solver's stream (instead of
 * spinning): for many solvers driven by more host threads than cores. */
#define SDR_SOLVER_BLOCKING_SYNC 1
/* The GPU is shared with other scenes (batches, the request server): every
 * pressure solve holds one SM instead of a cluster of them. Results are the
 * same either way. */
#define SDR_SOLVER_SHARED_GPU 2

/* Solver's public scalar fields (src/solver.rs:143-167) plus GPU-side counters. */
typedef struct {
    double time;
    uint64_t steps;
    uint64_t last_pcg_iters;
    uint64_t last_substeps;
    uint64_t particles;
    uint64_t drained;
    double last_residual;
    double emit_accum;
    uint64_t rng_state;
    uint64_t emitted;        /* particles injected since creation (mass-balance numerator) */
    uint64_t culled;         /* particles removed outside the outlet (wall tunnelling, out of domain) */
    uint64_t redistributed;  /* particle moves made by redistribution since creation */
    uint64_t nx, ny, nz;     /* MAC grid cells */
    double dx;
    sdr_vec3 origin;
    uint64_t particle_substeps; /* sum over substeps of the particles each one advanced */
    double device_ms;           /* device time of all substeps (CUDA events on the solver stream) */
    uint64_t substeps_total;    /* substeps run since creation */
} sdr_solver_stats;

/* Device time per phase group, accumulated while profiling is on (CUDA events
 * on the solver stream; milliseconds). pcg_cell_iters = sum over solves of
 * fluid cells x PCG iterations (the unit of the solve's algorithmic bytes). */
typedef struct {
    double emit_classify_sort_ms;
    double p2g_ms;
    double pressure_setup_ms;
    double pcg_ms;
    double gradient_extrapolate_ms;
    double g2p_advect_ms;
    double compact_ms;
    double redistribute_ms;
    uint64_t substeps;
    uint64_t pcg_launches;
    uint64_t pcg_cell_iters;
    uint64_t fluid_cells;       /* sum over solves of fluid cells */
    uint64_t particles;         /* sum over substeps of particles advanced */
    /* SM cycles inside the pressure-solve kernel by section: MIC(0) build,
     * forward+backward preconditioner sweeps, (unused), matvec, dot products,
     * update of p and r with the residual norm, search direction, setup/exit;
     * then per forward-sweep level: staging wait, compute, barrier, level
     * count; then the sum of sweep widths, of non-empty level ranges, and solves. */
    uint64_t pcg_section_cycles[16];
    /* redistribution: candidates (particles in over-cap cells) replayed, replay
     * sweeps run, and sweeps whose list was longer than the shared-memory one */
    uint64_t redist_candidates;
    uint64_t redist_sweeps;
    uint64_t redist_long_sweeps;
    uint64_t pcg_cluster_launches; /* solves that ran on the cluster kernel */
    /* bytes the substeps copied host -> device (emitted particles) and device
     * -> host (the per-substep status block) */
    uint64_t h2d_bytes;
    uint64_t d2h_bytes;
    uint64_t pcg_tile_launches; /* solves that ran on the whole-GPU tiled kernel */
    uint64_t redist_rounds;     /* decision rounds of long redistribution lists */
} sdr_profile;

/* FrameMetrics, src/metrics.rs:28-65 (counts as u64). */
typedef struct {
    uint64_t frame;
    double time_s;
    uint64_t particles;
    double fluid_volume_ml, drained_volume_ml, fill_fraction, wall_coverage;
    double mean_pressure_pa, max_pressure_pa, max_pressure_mmhg;
    double wall_pressure_pa, peak_wall_pressure_pa, peak_wall_pressure_mmhg;
    uint64_t membrane_artifacts;
    double max_speed_m_s, kinetic_energy;
    uint64_t pcg_iters;
} sdr_frame_metrics;

/* Summary, src/metrics.rs:69-97. */
typedef struct {
    uint64_t frames;
    double final_time_s, peak_fill_fraction, final_fill_fraction;
    double peak_wall_coverage, final_wall_coverage;
    double peak_membrane_pressure_pa, peak_membrane_pressure_mmhg;
    double mean_membrane_pressure_pa, mean_membrane_pressure_mmhg;
    double peak_pressure_pa, peak_pressure_mmhg;
    uint64_t membrane_artifacts_total;
    double total_drained_ml, injected_ml, mass_balance;
} sdr_summary;

typedef struct sdr_solver sdr_solver;
typedef struct sdr_metrics sdr_metrics;

/* ---------------------------------------------------------------- library */
int sdr_abi_version(void);
/* Thread-local message for the last failing call on this thread ("" if none). */
const char* sdr_last_error(void);
/* Number of kernel launches this library has issued in this process. */
uint64_t sdr_kernel_launch_count(void);

/* ---------------------------------------------------------------- solver */
/* Solver::new (src/solver.rs:184-222): grid covers the SDF bounds at sim_dx;
 * the static cavity mask is built on the device from the SDF. */
int sdr_solver_create(const sdr_sdf_desc* sdf, double sim_dx, const sdr_fluid_params* fluid,
                      const sdr_needle* needle, const sdr_solver_options* options,
                      sdr_solver** out);
int sdr_solver_destroy(sdr_solver* s);
/* Solver::outlet field (src/solver.rs:153); NULL removes the outlet. */
int sdr_solver_set_outlet(sdr_solver* s, const sdr_aabb* outlet_or_null);
/* Solver::solve field (src/solver.rs:154). */
int sdr_solver_set_solve_params(sdr_solver* s, const sdr_solve_params* params);
/* Solver::needle field (src/solver.rs:150). */
int sdr_solver_set_needle(sdr_solver* s, const sdr_needle* needle);
/* Solver::step (src/solver.rs:237-259): CFL sub-stepping with the dt/512 floor. */
int sdr_solver_step(sdr_solver* s, double dt);
/* Solver::substep (src/solver.rs:284-310). */
int sdr_solver_substep(sdr_solver* s, double dt);
/* Public fields time/steps/last_pcg_iters/last_substeps/drained (solver.rs:155-166). */
int sdr_solver_get_stats(const sdr_solver* s, sdr_solver_stats* out);
/* Solver::cfl_dt (src/solver.rs:262-281) for the current state, and the
 * MacGrid::max_speed (src/grid.rs:202-206) it uses: the face maxima the last
 * extrapolation sweep reduced on the device, combined on the host in f64.
 * Either output may be NULL. */
int sdr_solver_cfl(const sdr_solver* s, double* dt, double* grid_speed);
/* Entries of the redistribution candidate list (particles of over-cap cells
 * in one sweep of Solver::redistribute, src/solver.rs:454-557). 0 (default):
 * the particle capacity, which no sweep can exceed. A smaller list uses less
 * device memory; a sweep whose candidates do not fit moves nothing and the
 * substep returns SDR_ERR_CAPACITY (the error is reported once; the solver
 * stays usable). */
int sdr_solver_set_candidate_capacity(sdr_solver* s, uint64_t candidates);
/* Dot-product order inside the pressure solve. 1: the reference's order
 * (fixed 4096-cell chunks summed sequentially, partials in chunk order,
 * src/pressure.rs:588-603) — pressure and iteration counts then equal the
 * reference's bit for bit given the same right-hand side. 0 (default): a fixed
 * tree order (cells in wavefront order in 256-cell tiles, each added by a
 * fixed lane pattern and shuffle tree, the tiles likewise) — deterministic,
 * independent of the kernel and its CTA count, faster, differing from the
 * reference in the last bits of each dot. */
int sdr_solver_set_dot_order(sdr_solver* s, int reference_order);
/* Pressure-solve kernel. SDR_PCG_ONE_BLOCK: the MIC(0) wavefront sweeps on
 * one SM (lowest latency per level; the choice for small fluid regions), the
 * matvec, updates and dots on a cluster (sdr_solver_set_pcg_ctas).
 * SDR_PCG_CLUSTER: one thread-block cluster of up to 16 SMs, each level of
 * the sweeps spread over all of them (large fluid regions). Both run the same
 * per-cell arithmetic (pressure.rs:341-609) and the same dot orders, so they
 * give the same pressure bits (with the reference dot order, the
 * reference's). SDR_PCG_TILES: the whole GPU in one cooperative launch; the
 * grid's (j, k) lines cut into tiles of 16 x 16, one CTA per tile walking the
 * levels of its cells, tiles handing boundary values to their neighbours
 * through exchange entries that mark their own readiness (large fluid regions
 * on a GPU of their own; the cluster kernel if the device cannot launch it).
 * SDR_PCG_AUTO (default): from 200,000 fluid cells in the previous solve
 * (before the first solve: the particle count over particles_per_cell) the
 * tiled solve, or the cluster with SDR_SOLVER_SHARED_GPU; below that one
 * block. */
enum { SDR_PCG_AUTO = 0, SDR_PCG_ONE_BLOCK = 1, SDR_PCG_CLUSTER = 2, SDR_PCG_TILES = 3 };
int sdr_solver_set_pcg_kernel(sdr_solver* s, int kernel);
/* CTAs of the SDR_PCG_ONE_BLOCK solve's cluster (CTA 0 runs the sweeps).
 * 0 (default): 1 with SDR_SOLVER_SHARED_GPU, else 8 (or the largest cluster
 * the device schedules, if smaller). Results do not depend on it. */
int sdr_solver_set_pcg_ctas(sdr_solver* s, int ctas);
/* Phase-group timing with CUDA events (adds one event record per group):
 * on = 1. on = 2 also turns on the section timers inside the pressure-solve
 * kernel (pcg_section_cycles), which cost a little on its critical path. */
int sdr_solver_set_profiling(sdr_solver* s, int on);
int sdr_solver_get_profile(const sdr_solver* s, sdr_profile* out);
int sdr_solver_reset_profile(sdr_solver* s);
/* Restore the solver's scalar state (checkpoint / shadow stepping). */
int sdr_solver_set_scalars(sdr_solver* s, double time, double emit_accum, uint64_t steps,
                           uint64_t drained, uint64_t rng_state);
/* ParticleSet positions/velocities (src/particles.rs:13-16), widened to f64,
 * xyz interleaved; *n_out receives the particle count. SDR_ERR_BUFFER if cap < n. */
int sdr_solver_copy_particles(sdr_solver* s, double* pos_xyz, double* vel_xyz, size_t cap,
                              size_t* n_out);
/* Same, as the device's f32 storage (float xyz triples), e.g. for XYZ frame output. */
int sdr_solver_copy_particles_f32(sdr_solver* s, float* pos_xyz, float* vel_xyz, size_t cap,
                                  size_t* n_out);
/* Replace the particle set (values are rounded to f32 on the device). */
int sdr_solver_set_particles(sdr_solver* s, const double* pos_xyz, const double* vel_xyz,
                             size_t n);
/* Solver::pressure (src/solver.rs:164), nx*ny*nz f64. */
int sdr_solver_copy_pressure(sdr_solver* s, double* out, size_t cap);
/* Cell labels of the last classify (u8, SDR_CELL_*). */
int sdr_solver_copy_cells(sdr_solver* s, uint8_t* out, size_t cap);
/* Static cavity mask (src/solver.rs:173): 1 where the cell centre has phi < 0. */
int sdr_solver_copy_cavity_mask(sdr_solver* s, uint8_t* out, size_t cap);
/* MacGrid faces (src/grid.rs:92-100). which: 0 u, 1 v, 2 w, 3..5 the saved
 * (post-P2G) copies used by FLIP. f32 values widened to f64. */
int sdr_solver_copy_face(sdr_solver* s, int which, double* out, size_t cap);
int sdr_solver_set_face(sdr_solver* s, int which, const double* in, size_t n);
/* Diagnostics (src/solver.rs:763-890). */
int sdr_solver_max_pressure(sdr_solver* s, double* out);
int sdr_solver_mean_pressure(sdr_solver* s, double* out);
int sdr_solver_max_speed(sdr_solver* s, double* out);
int sdr_solver_cells_fluid_count(sdr_solver* s, uint64_t* out);
int sdr_solver_max_particles_per_cell(sdr_solver* s, uint64_t* out);
/* The P2G counting sort of the last substep: per-particle cell keys and the
 * stable permutation (sorted slot -> particle index), u32 each. */
int sdr_solver_copy_sort(sdr_solver* s, uint32_t* keys, uint32_t* perm, size_t cap,
                         size_t* n_out);

/* Phases of Solver::substep (src/solver.rs:284-310), for per-phase parity tests. */
enum {
    SDR_PHASE_EMIT = 0,
    SDR_PHASE_CLASSIFY = 1,
    SDR_PHASE_P2G = 2,        /* counting sort + gather; also saves the grid (save_grid) */
    SDR_PHASE_ADD_FORCES = 4, /* gravity on the working faces */
    SDR_PHASE_PROJECT = 5,    /* volume_source + project_capturing_with_source */
    SDR_PHASE_EXTRAPOLATE = 6,
    SDR_PHASE_G2P = 7,
    SDR_PHASE_ADVECT = 8,
    SDR_PHASE_BOUNDS = 9,
    SDR_PHASE_REDISTRIBUTE = 10,
    SDR_PHASE_CLOCK = 11
};
int sdr_solver_run_phase(sdr_solver* s, int phase, double dt);

/* ---------------------------------------------------------------- metrics */
/* MetricsCollector::new (src/metrics.rs:119-185): wall mask on the device. */
int sdr_metrics_create(sdr_solver* s, double cavity_volume, sdr_metrics** out);
int sdr_metrics_destroy(sdr_metrics* m);
/* MetricsCollector::record (src/metrics.rs:188-316): reductions on the device. */
int sdr_metrics_record(sdr_metrics* m, sdr_solver* s, uint64_t frame, sdr_frame_metrics* out);
/* MetricsCollector::summary (src/metrics.rs:324-382). */
int sdr_metrics_summary(const sdr_metrics* m, sdr_summary* out);
int sdr_metrics_wall_count(const sdr_metrics* m, uint64_t* out);

/* ---------------------------------------------------------------- geometry */
/* Grid of Sdf::from_mesh (src/sdf.rs:47-58) for triangles (9 f64 each). */
int sdr_sdf_mesh_grid(const double* tris, size_t ntri, double dx, double padding,
                      sdr_vec3* origin, uint64_t dims[3]);
/* Sdf::from_mesh_in_bounds values (src/sdf.rs:53-86, 187-272): winding-number
 * sign and closest-point distance per node, on the device. */
int sdr_sdf_from_mesh(const double* tris, size_t ntri, sdr_vec3 origin, double dx,
                      const uint64_t dims[3], double* out);
/* Test hook: the next sdr_sdf_from_mesh call on the calling thread makes one
 * bounded device wait run out on purpose, so that its error path runs without
 * any GPU fault. SDR_FAULT_SDF_STAGING: the bulk copy of the first triangle
 * tile is not issued, the staging wait gives up after its limit (about one
 * second), the kernel waits for its other copies in flight and reports, and
 * the call returns SDR_ERR_DEVICE_TIMEOUT. 0 clears a pending fault. */
enum { SDR_FAULT_NONE = 0, SDR_FAULT_SDF_STAGING = 1 };
int sdr_debug_inject(int fault);
/* Largest mesh sdr_sdf_from_mesh_noalloc accepts. */
#define SDR_NOALLOC_MAX_TRIANGLES 32768

/* The winding-number SDF of sdr_sdf_from_mesh for callers that cannot
 * allocate device memory: hosts that hand out their whole GPU memory budget
 * up front (a serving process that carves one pool at start-up and must not
 * grow), or latency-bound loops that cannot afford cudaMalloc's device
 * synchronisation. No counterpart in the reference (it has no device).
 *
 * tris_dev and out_dev are device pointers owned by the caller: ntri triangles
 * of 9 f64 (x0 y0 z0 x1 y1 z1 x2 y2 z2) and dims[0]*dims[1]*dims[2] f64 values
 * (x fastest, 8-byte aligned). stream is a cudaStream_t (NULL = the default
 * stream); the call returns after the work on it has finished.
 *
 * It calls no cudaMalloc/cudaFree: its scratch (the triangles padded to whole
 * staging tiles, ~2.4 MB, plus an error word) is a static device array that
 * every GPU loading this library holds until the process exits. Meshes with
 * more than SDR_NOALLOC_MAX_TRIANGLES triangles, and dims with a zero axis, an
 * axis above 2^31-1 or more than 2^37 nodes, return SDR_ERR_INVALID before
 * anything runs. The call is synchronous: it reads the kernel's error word
 * back and waits for the stream. The first call on a device looks up the
 * scratch's device address and caches it; do not use the library on a device
 * after a cudaDeviceReset of it in the same process. All calls share the one
 * scratch, which keeps the last call's contents, so calls that overlap on the
 * GPU (other streams, other host threads) race and must be serialised by the
 * caller. */
int sdr_sdf_from_mesh_noalloc(const double* tris_dev, size_t ntri, sdr_vec3 origin, double dx,
                              const uint64_t dims[3], double* out_dev, void* stream);

/* SinusParams, src/sinus.rs:26-45 (SI units). */
typedef struct {
    sdr_vec3 semi_axes;
    sdr_vec3 center;
    double taper;
    double bumpiness;
    double socket_x, socket_z;
    double socket_radius;
    double socket_depth;
    double model_dx;
} sdr_sinus_params;
/* Sdf::from_fn(SinusParams::implicit) (src/scene.rs:289-297, sinus.rs:89-119), on the device. */
int sdr_sdf_from_sinus(const sdr_sinus_params* p, sdr_vec3 origin, double dx,
                       const uint64_t dims[3], double* out);
/* |signed volume| of the naive-surface-nets mesh of a node field
 * (src/surface_nets.rs:48-195, src/mesh.rs:63-70): the parametric cavity volume. */
int sdr_surface_nets_volume(const double* values, const uint64_t dims[3], sdr_vec3 origin,
                            double dx, double* volume, uint64_t* triangles);

/* ---------------------------------------------------------------- frame output */
/* Particle files of src/output.rs: SDR_FORMAT_VTK is write_points_vtk
 * (output.rs:23-48, ASCII legacy VTK, numbers as Rust prints f64),
 * SDR_FORMAT_XYZ is write_points_xyz (output.rs:98-110, raw little-endian f32
 * triples). */
enum { SDR_FORMAT_VTK = 0, SDR_FORMAT_XYZ = 1 };
/* n points from host memory, xyz interleaved. */
/* ---------------------------------------------------------------- previews
 * src/render.rs. SlicePlane (render.rs:45-56): in-plane horizontal and
 * vertical axes, the axis sliced along (0 = x, 1 = y, 2 = z), the slice
 * coordinate and the half-thickness of the particle band, whether larger
 * vertical coordinates go up (flip_v), a silhouette projection instead of a
 * slice, and the amber pool instead of speed-coloured dots. */
typedef struct {
    int32_t hax, vax, oax, flip_v, project, amber;
    double slice, slab;
} sdr_slice_plane;
/* SlicePlane::xy / xz / yz / projected_along_gravity (render.rs:64-136). */
int sdr_slice_plane_xy(double slice, double slab, sdr_slice_plane* out);
int sdr_slice_plane_xz(double slice, double slab, sdr_slice_plane* out);
int sdr_slice_plane_yz(double slice, double slab, sdr_slice_plane* out);
int sdr_slice_plane_gravity(sdr_vec3 gravity, sdr_slice_plane* out);
/* render_slice (render.rs:139-236) of the solver's current state, drawn on
 * the device: RGB8 rows top to bottom into rgb (cap bytes, at least
 * 3 * w * h; w and h are written first, so a call with rgb = NULL returns
 * SDR_ERR_BUFFER with the size). vmax <= 0 scales speed to the peak. */
int sdr_render_slice(sdr_solver* s, const sdr_slice_plane* plane, uint32_t target_px, double vmax, uint8_t* rgb,
                     size_t cap, uint32_t* w, uint32_t* h);
/* render_timeseries (render.rs:351-406) of a run's frames. */
int sdr_render_timeseries(const sdr_frame_metrics* frames, size_t n, uint32_t w, uint32_t h, uint8_t* rgb,
                          size_t cap);
/* save_png (render.rs:409-414): 8-bit RGB PNG. */
int sdr_write_png(const char* path, const uint8_t* rgb, uint32_t w, uint32_t h);

/* Metrics files. serde_json's to_string_pretty layout: shortest round-trip
 * digits for every f64 (plain notation with at least one fractional digit for
 * 1e-5 <= |v| < 1e16, else d.ddde[-]x; null if not finite), two-space indent.
 * MetricsCollector::write_json (src/metrics.rs:385-391): the frames as a JSON array. */
int sdr_metrics_write_json(const sdr_metrics* m, const char* path);
/* MetricsCollector::write_csv (src/metrics.rs:394-431): header + one row per
 * frame, each value as Rust's `{}` prints it. */
int sdr_metrics_write_csv(const sdr_metrics* m, const char* path);
/* The same two files from a caller's array of frames. */
int sdr_frames_write_json(const sdr_frame_metrics* frames, size_t n, const char* path);
int sdr_frames_write_csv(const sdr_frame_metrics* frames, size_t n, const char* path);
/* summary.json of cmd_simulate (src/main.rs:306-310). */
int sdr_summary_write_json(const sdr_summary* summary, const char* path);

int sdr_write_points(const char* path, int32_t format, const float* xyz, size_t n);
/* frame_path (output.rs:114-122): "<dir>/<prefix>_<frame, 6 digits>.<vtk|xyz>". */
int sdr_frame_path(const char* dir, const char* prefix, uint64_t frame, int32_t format, char* out, size_t cap);

/* The per-frame output of cmd_simulate (main.rs:255-266) without stopping the
 * solver: submit copies the current positions to one of two pinned host
 * buffers on the solver's stream and returns; a writer thread waits for that
 * copy and writes frame_path(dir, prefix, frame, format) while the next frames
 * run. A third submit waits for the older buffer's file to be written. The
 * directory must exist. Write errors are reported by the next submit, flush
 * or destroy. */
typedef struct sdr_frame_writer sdr_frame_writer;
int sdr_frame_writer_create(const char* dir, const char* prefix, int32_t format, sdr_frame_writer** out);
int sdr_frame_writer_submit(sdr_frame_writer* w, sdr_solver* s, uint64_t frame);
/* Waits until every submitted frame is on disk. */
int sdr_frame_writer_flush(sdr_frame_writer* w);
int sdr_frame_writer_destroy(sdr_frame_writer* w);

/* ---------------------------------------------------------------- batches and serving
 * Many independent scenes on one GPU. The reference runs one scene per
 * process (main.rs:215-386: build the scene, Solver::step per frame,
 * MetricsCollector::record, summary); these entry points run that same loop
 * for many scenes at once, each scene on its own solver, CUDA stream and host
 * thread, so the scenes' kernels (one SM per pressure solve) share the GPU.
 * A scene's result does not depend on what runs beside it. */

/* One scene: the solver set-up of Solver::new plus the run length and the
 * cavity volume the metrics need (scene.rs:312). The SDF data is copied when
 * the scene is handed over. */
typedef struct {
    sdr_sdf_desc sdf;
    double sim_dx;
    sdr_fluid_params fluid;
    sdr_needle needle;
    sdr_solve_params solve;
    int32_t has_outlet;
    int32_t reserved0;
    sdr_aabb outlet;
    double cavity_volume;   /* m^3 */
    double frame_dt;        /* seconds per frame */
    uint64_t frames;        /* frames to run */
    uint64_t max_particles; /* device particle capacity (0 = derive from the dose) */
} sdr_scene_desc;

/* Device bytes a scene needs while it runs (grid, particle capacity, SDF,
 * workspace): the admission estimate of the server. Host arithmetic only. */
int sdr_scene_footprint(const sdr_scene_desc* scene, uint64_t* bytes);

typedef struct sdr_batch sdr_batch;
int sdr_batch_create(const sdr_scene_desc* scenes, size_t n, int32_t device, sdr_batch** out);
/* Run every scene of the batch to its frame count with up to `concurrency`
 * scenes in flight (0 = all; 1 = one after another, each on a default solver
 * as sdr_solver_create makes it: the plain path). Concurrent scenes run with
 * SDR_SOLVER_SHARED_GPU. Scene
 * failures are reported per scene by sdr_batch_result; the call itself fails
 * only for bad arguments. */
int sdr_batch_run(sdr_batch* b, uint32_t concurrency);
/* The batch's scenes packed together (no counterpart in the reference, which
 * runs one scene per process): every packed step advances each live scene by
 * one substep at its own CFL step, and each operation of the substep is ONE
 * launch for all of them - a ragged offset table gives every scene its share
 * of the launch's blocks, and a persistent grid walks them running the
 * operation's kernel body with that scene's arguments (each scene's pressure
 * solve is one block, which runs to that scene's own convergence). Scenes
 * leave as they finish their frames. Every scene computes exactly what it
 * computes alone, so results equal sdr_batch_run's bit for bit. Scene times
 * (sdr_batch_result's seconds) run from the start of the call to the scene's
 * last frame. */
int sdr_batch_run_packed(sdr_batch* b);
/* Of the last sdr_batch_run_packed: kernel launches, packed steps, CUDA-graph
 * captures (a packed step is captured as one graph and replayed while its
 * launch plan - the operations, the scenes in each and their grid sizes,
 * rounded up to powers of two - is unchanged) and the CTAs per SM the
 * autotuner chose for the persistent grids (it times 2, 4, 8 and 16 CTAs per
 * SM over the first packed steps and keeps the fastest by particle-substeps
 * per second; 0 if the run was too short to finish tuning). Either of the last
 * two may be NULL. */
int sdr_batch_packed_counters(const sdr_batch* b, uint64_t* launches, uint64_t* steps, uint64_t* graph_captures,
                              int32_t* ctas_per_sm);
/* status: SDR_OK or the scene's error code (message in `error`, may be NULL). */
int sdr_batch_result(const sdr_batch* b, size_t i, int32_t* status, sdr_summary* summary,
                     sdr_solver_stats* stats_or_null, double* seconds_or_null, char* error, size_t error_cap);
int sdr_batch_destroy(sdr_batch* b);

/* A request loop: scenes submitted at any time are admitted in arrival order
 * while their footprint fits the byte budget and a slot is free, run
 * concurrently, and release their memory when their summary is ready. */
typedef struct sdr_server sdr_server;
enum { SDR_REQ_QUEUED = 0, SDR_REQ_RUNNING = 1, SDR_REQ_DONE = 2, SDR_REQ_FAILED = 3 };
typedef struct {
    uint64_t submitted, completed, failed;
    uint32_t active, peak_active;
    uint64_t bytes_in_use, peak_bytes;
} sdr_server_stats;
int sdr_server_create(int32_t device, uint64_t budget_bytes, uint32_t max_active, sdr_server** out);
/* The same request loop with every admitted scene in one packed engine
 * (sdr_batch_run_packed): requests join the packed steps as slots and budget
 * free up and leave when their summary is ready - continuous batching on one
 * host thread and one stream. */
int sdr_server_create_packed(int32_t device, uint64_t budget_bytes, uint32_t max_active, sdr_server** out);
int sdr_server_submit(sdr_server* s, const sdr_scene_desc* scene, uint64_t* ticket);
/* state: SDR_REQ_*. When done: the summary and the seconds from submission to
 * summary (time-to-summary); when failed: the message in `error` (may be NULL). */
int sdr_server_poll(sdr_server* s, uint64_t ticket, int32_t* state, sdr_summary* summary_or_null,
                    double* seconds_or_null, char* error, size_t error_cap);
int sdr_server_get_stats(sdr_server* s, sdr_server_stats* out);
/* Waits for every admitted and queued request, then frees the server. */
int sdr_server_destroy(sdr_server* s);

#ifdef __cplusplus
}
#endif
#endif /* SDR_GPU_H */
