"""ctypes binding of libsdr_gpu.so (the C ABI in include/sdr_gpu.h).

The library is the product: every compute entry point runs CUDA kernels on
the device. Loading fails loudly if the in-tree library is missing; there is
no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsdr_gpu.so")

SDR_OK = 0
(SDR_ERR_INVALID, SDR_ERR_CUDA, SDR_ERR_OOM, SDR_ERR_CAPACITY, SDR_ERR_DEVICE_TIMEOUT, SDR_ERR_NO_DEVICE,
 SDR_ERR_BUFFER, SDR_ERR_IO) = range(1, 9)
NOALLOC_MAX_TRIANGLES = 32768
ERRORS = {1: "INVALID", 2: "CUDA", 3: "OOM", 4: "CAPACITY", 5: "DEVICE_TIMEOUT", 6: "NO_DEVICE", 7: "BUFFER"}

PHASE_EMIT, PHASE_CLASSIFY, PHASE_P2G, PHASE_ADD_FORCES = 0, 1, 2, 4
PHASE_PROJECT, PHASE_EXTRAPOLATE, PHASE_G2P, PHASE_ADVECT = 5, 6, 7, 8
PHASE_BOUNDS, PHASE_REDISTRIBUTE, PHASE_CLOCK = 9, 10, 11


class SdrError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"sdr error {ERRORS.get(code, code)}: {msg}")
        self.code = code


class Vec3(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double)]


class Aabb(C.Structure):
    _fields_ = [("min", Vec3), ("max", Vec3)]


class FluidParamsC(C.Structure):
    _fields_ = [("density", C.c_double), ("gravity", Vec3), ("flip_ratio", C.c_double),
                ("particles_per_cell", C.c_uint64), ("volume_stiffness", C.c_double),
                ("redistribute", C.c_int32), ("reserved0", C.c_int32), ("redist_cap_factor", C.c_double)]


class NeedleC(C.Structure):
    _fields_ = [("tip", Vec3), ("axis", Vec3), ("radius", C.c_double), ("flow_rate", C.c_double),
                ("inject_until", C.c_double)]


class SolveParamsC(C.Structure):
    _fields_ = [("max_iters", C.c_uint64), ("tol", C.c_double)]


class SdfDesc(C.Structure):
    _fields_ = [("origin", Vec3), ("dx", C.c_double), ("nx", C.c_uint64), ("ny", C.c_uint64),
                ("nz", C.c_uint64), ("data", C.POINTER(C.c_double))]


class SolverOptions(C.Structure):
    _fields_ = [("max_particles", C.c_uint64), ("device", C.c_int32), ("flags", C.c_int32)]


SOLVER_BLOCKING_SYNC = 1
SOLVER_SHARED_GPU = 2
PCG_AUTO, PCG_ONE_BLOCK, PCG_CLUSTER, PCG_TILES = 0, 1, 2, 3


class SolverStats(C.Structure):
    _fields_ = [("time", C.c_double), ("steps", C.c_uint64), ("last_pcg_iters", C.c_uint64),
                ("last_substeps", C.c_uint64), ("particles", C.c_uint64), ("drained", C.c_uint64),
                ("last_residual", C.c_double), ("emit_accum", C.c_double), ("rng_state", C.c_uint64),
                ("emitted", C.c_uint64), ("culled", C.c_uint64), ("redistributed", C.c_uint64),
                ("nx", C.c_uint64), ("ny", C.c_uint64), ("nz", C.c_uint64), ("dx", C.c_double),
                ("origin", Vec3), ("particle_substeps", C.c_uint64), ("device_ms", C.c_double),
                ("substeps_total", C.c_uint64)]


class Profile(C.Structure):
    _fields_ = [("emit_classify_sort_ms", C.c_double), ("p2g_ms", C.c_double), ("pressure_setup_ms", C.c_double),
                ("pcg_ms", C.c_double), ("gradient_extrapolate_ms", C.c_double), ("g2p_advect_ms", C.c_double),
                ("compact_ms", C.c_double), ("redistribute_ms", C.c_double), ("substeps", C.c_uint64),
                ("pcg_launches", C.c_uint64), ("pcg_cell_iters", C.c_uint64), ("fluid_cells", C.c_uint64),
                ("particles", C.c_uint64), ("pcg_section_cycles", C.c_uint64 * 16),
                ("redist_candidates", C.c_uint64), ("redist_sweeps", C.c_uint64),
                ("redist_long_sweeps", C.c_uint64), ("pcg_cluster_launches", C.c_uint64),
                ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64), ("pcg_tile_launches", C.c_uint64),
                ("redist_rounds", C.c_uint64)]

    def to_dict(self):
        d = {n: getattr(self, n) for n, _ in self._fields_}
        d["pcg_section_cycles"] = list(self.pcg_section_cycles)
        return d


class SlicePlaneC(C.Structure):
    _fields_ = [("hax", C.c_int32), ("vax", C.c_int32), ("oax", C.c_int32), ("flip_v", C.c_int32),
                ("project", C.c_int32), ("amber", C.c_int32), ("slice", C.c_double), ("slab", C.c_double)]


_FM = ["frame:u", "time_s", "particles:u", "fluid_volume_ml", "drained_volume_ml", "fill_fraction",
       "wall_coverage", "mean_pressure_pa", "max_pressure_pa", "max_pressure_mmhg", "wall_pressure_pa",
       "peak_wall_pressure_pa", "peak_wall_pressure_mmhg", "membrane_artifacts:u", "max_speed_m_s",
       "kinetic_energy", "pcg_iters:u"]
_SM = ["frames:u", "final_time_s", "peak_fill_fraction", "final_fill_fraction", "peak_wall_coverage",
       "final_wall_coverage", "peak_membrane_pressure_pa", "peak_membrane_pressure_mmhg",
       "mean_membrane_pressure_pa", "mean_membrane_pressure_mmhg", "peak_pressure_pa",
       "peak_pressure_mmhg", "membrane_artifacts_total:u", "total_drained_ml", "injected_ml",
       "mass_balance"]


def _fields(spec):
    return [(n.split(":")[0], C.c_uint64 if n.endswith(":u") else C.c_double) for n in spec]


class FrameMetricsC(C.Structure):
    _fields_ = _fields(_FM)

    def to_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class SummaryC(C.Structure):
    _fields_ = _fields(_SM)

    def to_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class SinusParamsC(C.Structure):
    _fields_ = [("semi_axes", Vec3), ("center", Vec3), ("taper", C.c_double), ("bumpiness", C.c_double),
                ("socket_x", C.c_double), ("socket_z", C.c_double), ("socket_radius", C.c_double),
                ("socket_depth", C.c_double), ("model_dx", C.c_double)]


class SceneDesc(C.Structure):
    _fields_ = [("sdf", SdfDesc), ("sim_dx", C.c_double), ("fluid", FluidParamsC), ("needle", NeedleC),
                ("solve", SolveParamsC), ("has_outlet", C.c_int32), ("reserved0", C.c_int32), ("outlet", Aabb),
                ("cavity_volume", C.c_double), ("frame_dt", C.c_double), ("frames", C.c_uint64),
                ("max_particles", C.c_uint64)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("active", C.c_uint32), ("peak_active", C.c_uint32), ("bytes_in_use", C.c_uint64),
                ("peak_bytes", C.c_uint64)]

    def to_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED = 0, 1, 2, 3
FORMAT_VTK, FORMAT_XYZ = 0, 1
FAULT_NONE, FAULT_SDF_STAGING = 0, 1

P = C.POINTER
d, u64, i32, vp, sz = C.c_double, C.c_uint64, C.c_int, C.c_void_p, C.c_size_t

# (restype, argtypes) for every entry point declared in include/sdr_gpu.h.
SIGNATURES = {
    "sdr_abi_version": (i32, []),
    "sdr_last_error": (C.c_char_p, []),
    "sdr_kernel_launch_count": (u64, []),
    "sdr_solver_create": (i32, [P(SdfDesc), d, P(FluidParamsC), P(NeedleC), P(SolverOptions), P(vp)]),
    "sdr_solver_destroy": (i32, [vp]),
    "sdr_solver_set_outlet": (i32, [vp, P(Aabb)]),
    "sdr_solver_set_solve_params": (i32, [vp, P(SolveParamsC)]),
    "sdr_solver_set_needle": (i32, [vp, P(NeedleC)]),
    "sdr_solver_step": (i32, [vp, d]),
    "sdr_solver_substep": (i32, [vp, d]),
    "sdr_solver_get_stats": (i32, [vp, P(SolverStats)]),
    "sdr_solver_set_scalars": (i32, [vp, d, d, u64, u64, u64]),
    "sdr_solver_cfl": (i32, [vp, P(d), P(d)]),
    "sdr_solver_set_candidate_capacity": (i32, [vp, u64]),
    "sdr_debug_inject": (i32, [i32]),
    "sdr_solver_set_dot_order": (i32, [vp, i32]),
    "sdr_solver_set_pcg_kernel": (i32, [vp, i32]),
    "sdr_solver_set_pcg_ctas": (i32, [vp, i32]),
    "sdr_solver_set_profiling": (i32, [vp, i32]),
    "sdr_solver_get_profile": (i32, [vp, P(Profile)]),
    "sdr_solver_reset_profile": (i32, [vp]),
    "sdr_solver_copy_particles": (i32, [vp, P(d), P(d), sz, P(sz)]),
    "sdr_solver_copy_particles_f32": (i32, [vp, P(C.c_float), P(C.c_float), sz, P(sz)]),
    "sdr_solver_set_particles": (i32, [vp, P(d), P(d), sz]),
    "sdr_solver_copy_pressure": (i32, [vp, P(d), sz]),
    "sdr_solver_copy_cells": (i32, [vp, P(C.c_uint8), sz]),
    "sdr_solver_copy_cavity_mask": (i32, [vp, P(C.c_uint8), sz]),
    "sdr_solver_copy_face": (i32, [vp, i32, P(d), sz]),
    "sdr_solver_set_face": (i32, [vp, i32, P(d), sz]),
    "sdr_solver_max_pressure": (i32, [vp, P(d)]),
    "sdr_solver_mean_pressure": (i32, [vp, P(d)]),
    "sdr_solver_max_speed": (i32, [vp, P(d)]),
    "sdr_solver_cells_fluid_count": (i32, [vp, P(u64)]),
    "sdr_solver_max_particles_per_cell": (i32, [vp, P(u64)]),
    "sdr_solver_copy_sort": (i32, [vp, P(C.c_uint32), P(C.c_uint32), sz, P(sz)]),
    "sdr_solver_run_phase": (i32, [vp, i32, d]),
    "sdr_metrics_create": (i32, [vp, d, P(vp)]),
    "sdr_metrics_destroy": (i32, [vp]),
    "sdr_metrics_record": (i32, [vp, vp, u64, P(FrameMetricsC)]),
    "sdr_metrics_summary": (i32, [vp, P(SummaryC)]),
    "sdr_metrics_wall_count": (i32, [vp, P(u64)]),
    "sdr_sdf_mesh_grid": (i32, [P(d), sz, d, d, P(Vec3), P(u64)]),
    "sdr_sdf_from_mesh": (i32, [P(d), sz, Vec3, d, P(u64), P(d)]),
    "sdr_sdf_from_sinus": (i32, [P(SinusParamsC), Vec3, d, P(u64), P(d)]),
    "sdr_sdf_from_mesh_noalloc": (i32, [vp, sz, Vec3, d, P(u64), vp, vp]),
    "sdr_surface_nets_volume": (i32, [P(d), P(u64), Vec3, d, P(d), P(u64)]),
    "sdr_write_points": (i32, [C.c_char_p, C.c_int32, P(C.c_float), sz]),
    "sdr_metrics_write_json": (i32, [vp, C.c_char_p]),
    "sdr_slice_plane_xy": (i32, [d, d, P(SlicePlaneC)]),
    "sdr_slice_plane_xz": (i32, [d, d, P(SlicePlaneC)]),
    "sdr_slice_plane_yz": (i32, [d, d, P(SlicePlaneC)]),
    "sdr_slice_plane_gravity": (i32, [Vec3, P(SlicePlaneC)]),
    "sdr_render_slice": (i32, [vp, P(SlicePlaneC), C.c_uint32, d, P(C.c_uint8), sz, P(C.c_uint32), P(C.c_uint32)]),
    "sdr_render_timeseries": (i32, [P(FrameMetricsC), sz, C.c_uint32, C.c_uint32, P(C.c_uint8), sz]),
    "sdr_write_png": (i32, [C.c_char_p, P(C.c_uint8), C.c_uint32, C.c_uint32]),
    "sdr_metrics_write_csv": (i32, [vp, C.c_char_p]),
    "sdr_frames_write_json": (i32, [P(FrameMetricsC), sz, C.c_char_p]),
    "sdr_frames_write_csv": (i32, [P(FrameMetricsC), sz, C.c_char_p]),
    "sdr_summary_write_json": (i32, [P(SummaryC), C.c_char_p]),
    "sdr_frame_path": (i32, [C.c_char_p, C.c_char_p, u64, C.c_int32, C.c_char_p, sz]),
    "sdr_frame_writer_create": (i32, [C.c_char_p, C.c_char_p, C.c_int32, P(vp)]),
    "sdr_frame_writer_submit": (i32, [vp, vp, u64]),
    "sdr_frame_writer_flush": (i32, [vp]),
    "sdr_frame_writer_destroy": (i32, [vp]),
    "sdr_scene_footprint": (i32, [P(SceneDesc), P(u64)]),
    "sdr_batch_create": (i32, [P(SceneDesc), sz, C.c_int32, P(vp)]),
    "sdr_batch_run": (i32, [vp, C.c_uint32]),
    "sdr_batch_result": (i32, [vp, sz, P(C.c_int32), P(SummaryC), P(SolverStats), P(d), C.c_char_p, sz]),
    "sdr_batch_destroy": (i32, [vp]),
    "sdr_batch_run_packed": (i32, [vp]),
    "sdr_batch_packed_counters": (i32, [vp, P(u64), P(u64), P(u64), P(C.c_int32)]),
    "sdr_server_create_packed": (i32, [C.c_int32, u64, C.c_uint32, P(vp)]),
    "sdr_server_create": (i32, [C.c_int32, u64, C.c_uint32, P(vp)]),
    "sdr_server_submit": (i32, [vp, P(SceneDesc), P(u64)]),
    "sdr_server_poll": (i32, [vp, u64, P(C.c_int32), P(SummaryC), P(d), C.c_char_p, sz]),
    "sdr_server_get_stats": (i32, [vp, P(ServerStats)]),
    "sdr_server_destroy": (i32, [vp]),
}

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load the in-tree library (build it first with ``python -m sdr_b200.build``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise ImportError(f"{path} is missing: build it with `python -m sdr_b200.build` "
                              "(the CUDA path has no CPU fallback)")
        lib = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def check(code: int) -> None:
    if code != SDR_OK:
        msg = load().sdr_last_error()
        raise SdrError(code, msg.decode() if msg else "")
