/*
 * sdr oracle: C ABI of the CPU restatement of uselessgoddess/sdr's FLIP/PIC substep.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker for the CUDA path in
 * sdr_b200/. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it. It is never linked into, or called by, the product.
 *
 * Everything is f64, in the reference's operation order (src/math.rs:1-6).
 * Cell labels use the product's encoding: 0 = Solid, 1 = Fluid, 2 = Air
 * (src/pressure.rs:24-32).
 */
#ifndef SDR_ORACLE_H
#define SDR_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_solver orc_solver;
typedef struct orc_metrics orc_metrics;

/* FluidParams, src/solver.rs:41-71 */
typedef struct {
    double density;
    double gravity[3];
    double flip_ratio;
    uint64_t particles_per_cell;
    double volume_stiffness;
    int32_t redistribute;
    int32_t _pad;
    double redist_cap_factor;
} orc_fluid;

/* Needle, src/solver.rs:89-103 */
typedef struct {
    double tip[3];
    double axis[3];
    double radius;
    double flow_rate;
    double inject_until;
} orc_needle;

/* SinusParams, src/sinus.rs:26-45 */
typedef struct {
    double semi_axes[3];
    double center[3];
    double taper;
    double bumpiness;
    double socket_xz[2];
    double socket_radius;
    double socket_depth;
    double model_dx;
} orc_sinus;

/* FrameMetrics, src/metrics.rs:28-65 (counts widened to u64) */
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
} orc_frame_metrics;

/* Summary, src/metrics.rs:69-97 */
typedef struct {
    uint64_t frames;
    double final_time_s, peak_fill_fraction, final_fill_fraction;
    double peak_wall_coverage, final_wall_coverage;
    double peak_membrane_pressure_pa, peak_membrane_pressure_mmhg;
    double mean_membrane_pressure_pa, mean_membrane_pressure_mmhg;
    double peak_pressure_pa, peak_pressure_mmhg;
    uint64_t membrane_artifacts_total;
    double total_drained_ml, injected_ml, mass_balance;
} orc_summary;

/* Substep phases, in the order of Solver::substep (src/solver.rs:284-310). */
enum {
    ORC_PHASE_EMIT = 0,
    ORC_PHASE_CLASSIFY = 1,
    ORC_PHASE_P2G = 2,
    ORC_PHASE_SAVE_GRID = 3,
    ORC_PHASE_ADD_FORCES = 4,
    ORC_PHASE_PROJECT = 5, /* volume_source + project_capturing_with_source */
    ORC_PHASE_EXTRAPOLATE = 6,
    ORC_PHASE_G2P = 7,
    ORC_PHASE_ADVECT = 8,
    ORC_PHASE_BOUNDS = 9,
    ORC_PHASE_REDISTRIBUTE = 10,
    ORC_PHASE_CLOCK = 11 /* time += dt; steps += 1 */
};

void orc_set_threads(int n);
int orc_get_threads(void);

/* ---- geometry (src/sdf.rs, src/sinus.rs, src/surface_nets.rs, src/mesh.rs) ---- */
double orc_point_triangle_distance_sq(const double p[3], const double a[3], const double b[3],
                                      const double c[3]);
double orc_signed_distance_to_mesh(const double p[3], const double* tris, size_t ntri);
/* Grid of Sdf::from_mesh (sdf.rs:47-58): fills origin and dims. */
void orc_sdf_mesh_grid(const double* tris, size_t ntri, double dx, double padding,
                       double origin[3], uint64_t dims[3]);
void orc_sdf_from_mesh(const double* tris, size_t ntri, const double origin[3], double dx,
                       const uint64_t dims[3], double* out);
double orc_sinus_implicit(const orc_sinus* s, const double p[3]);
void orc_sinus_bounds(const orc_sinus* s, double mn[3], double mx[3]);
double orc_sinus_socket_bottom_y(const orc_sinus* s);
void orc_sinus_suggested_needle(const orc_sinus* s, double tip[3], double axis[3]);
/* Sdf::from_fn(implicit) over explicit grid (scene.rs:289-297). */
void orc_sdf_from_sinus(const orc_sinus* s, const double origin[3], double dx,
                        const uint64_t dims[3], double* out);
/* Surface nets mesh of the implicit (sinus.rs:141-150) -> |signed volume| and triangle count. */
double orc_sinus_mesh_volume(const orc_sinus* s, uint64_t* ntri_out);
/* Surface nets of the implicit; copies triangles (9 doubles each) if out != NULL and cap fits. */
size_t orc_sinus_mesh(const orc_sinus* s, double* tris_out, size_t cap_tris);
double orc_mesh_signed_volume(const double* tris, size_t ntri);
double orc_sdf_sample(const double* data, const uint64_t dims[3], const double origin[3],
                      double dx, const double p[3]);
void orc_sdf_gradient(const double* data, const uint64_t dims[3], const double origin[3],
                      double dx, const double p[3], double g[3]);

/* ---- solver (src/solver.rs) ---- */
orc_solver* orc_solver_new(const double* sdf_data, const uint64_t sdf_dims[3],
                           const double sdf_origin[3], double sdf_dx, double sim_dx,
                           const orc_fluid* fluid, const orc_needle* needle);
void orc_solver_free(orc_solver* s);
void orc_solver_set_outlet(orc_solver* s, int has, const double mn[3], const double mx[3]);
void orc_solver_set_solve(orc_solver* s, uint64_t max_iters, double tol);
void orc_solver_set_needle(orc_solver* s, const orc_needle* needle);
void orc_solver_step(orc_solver* s, double dt);
void orc_solver_substep(orc_solver* s, double dt);
void orc_solver_phase(orc_solver* s, int phase, double dt);
double orc_solver_cfl_dt(const orc_solver* s);
void orc_solver_grid(const orc_solver* s, uint64_t dims[3], double origin[3], double* dx);
size_t orc_solver_num_particles(const orc_solver* s);
void orc_solver_get_particles(const orc_solver* s, double* pos, double* vel);
void orc_solver_set_particles(orc_solver* s, size_t n, const double* pos, const double* vel);
/* scalars: time, emit_accum (f64); steps, last_pcg_iters, last_substeps, drained, rng (u64) */
void orc_solver_get_scalars(const orc_solver* s, double* time, double* emit_accum,
                            uint64_t* steps, uint64_t* last_pcg_iters, uint64_t* last_substeps,
                            uint64_t* drained, uint64_t* rng);
void orc_solver_set_scalars(orc_solver* s, double time, double emit_accum, uint64_t steps,
                            uint64_t drained, uint64_t rng);
/* which: 0 u, 1 v, 2 w, 3 saved_u, 4 saved_v, 5 saved_w */
void orc_solver_get_face(const orc_solver* s, int which, double* out);
void orc_solver_set_face(orc_solver* s, int which, const double* in);
void orc_solver_get_cells(const orc_solver* s, uint8_t* out);
void orc_solver_set_cells(orc_solver* s, const uint8_t* in);
void orc_solver_get_cavity_mask(const orc_solver* s, uint8_t* out);
void orc_solver_get_pressure(const orc_solver* s, double* out);
void orc_solver_get_source(const orc_solver* s, double dt, double* out);
double orc_solver_max_pressure(const orc_solver* s);
double orc_solver_mean_pressure(const orc_solver* s);
double orc_solver_max_speed(const orc_solver* s);
double orc_solver_kinetic_energy(const orc_solver* s);
uint64_t orc_solver_max_particles_per_cell(const orc_solver* s);
uint64_t orc_solver_cells_fluid_count(const orc_solver* s);
double orc_solver_grid_max_speed(const orc_solver* s);
/* Per-substep phase timers accumulated since the last reset, seconds (diagnostic). */
void orc_solver_phase_times(const orc_solver* s, double out[12]);

/* ---- pressure (src/pressure.rs) on caller arrays ---- */
/* u,v,w modified in place; cells u8 labels; source may be NULL. Returns iterations. */
uint64_t orc_project(uint64_t nx, uint64_t ny, uint64_t nz, double dx, double* u, double* v,
                     double* w, const uint8_t* cells, double rho, double dt, uint64_t max_iters,
                     double tol, const double* source, double* pressure_out, double* residual_out);
/* The MIC(0) factor (pressure.rs:442-513) for a label field. */
void orc_build_mic0(uint64_t nx, uint64_t ny, uint64_t nz, const uint8_t* cells, double* precon);
/* One preconditioner application z = M^-1 r (pressure.rs:517-570). */
void orc_apply_mic0(uint64_t nx, uint64_t ny, uint64_t nz, const uint8_t* cells,
                    const double* precon, const double* r, double* z);
double orc_dot(const double* a, const double* b, size_t n);

/* ---- metrics (src/metrics.rs) ---- */
orc_metrics* orc_metrics_new(const orc_solver* s, double cavity_volume);
void orc_metrics_free(orc_metrics* m);
void orc_metrics_record(orc_metrics* m, const orc_solver* s, uint64_t frame,
                        orc_frame_metrics* out);
void orc_metrics_summary(const orc_metrics* m, orc_summary* out);
uint64_t orc_metrics_wall_count(const orc_metrics* m);
void orc_metrics_get_masks(const orc_metrics* m, uint8_t* is_wall, uint8_t* washed);
void orc_membrane_stats(const double* values, size_t n, double cap, double* mean, double* peak,
                        uint64_t* artifacts);
/* hash_jitter (solver.rs:916-930) */
void orc_hash_jitter(uint64_t key, double out[3]);

/* ---- render (src/render.rs) into RGB8 buffers of w*h*3 bytes ---- */
typedef struct {
    int32_t hax, vax, oax, flip_v, project, amber;
    double slice, slab;
} orc_slice_plane;
void orc_render_slice_dims(const orc_solver* s, const orc_slice_plane* p, uint32_t target_px, uint32_t* w,
                           uint32_t* h);
void orc_render_slice(const orc_solver* s, const orc_slice_plane* p, uint32_t target_px, double vmax,
                      uint8_t* rgb);
void orc_render_timeseries(const orc_frame_metrics* frames, size_t n, uint32_t w, uint32_t h, uint8_t* rgb);

#ifdef __cplusplus
}
#endif
#endif
