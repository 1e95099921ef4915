"""Python mirror of the reference's solver-facing API over the C ABI.

``Solver`` follows ``Solver`` in uselessgoddess/sdr ``src/solver.rs:143-890``
(``step``, ``substep``, ``particle_volume``, ``fluid_volume``, ``drained_volume``,
``max_pressure`` ...), ``MetricsCollector`` follows ``src/metrics.rs:102-431``,
and ``build_scene`` follows ``SceneConfig::build`` (``src/scene.rs:266-334``)
with the SDF voxelised on the device. Every call goes through
``libsdr_gpu.so``; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib
from ._lib import check
from .scene import FluidParams, Needle, ResolvedScene, SceneConfig, SinusParams, SolveParams, load_mesh, MM


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _v3(x) -> _lib.Vec3:
    return _lib.Vec3(float(x[0]), float(x[1]), float(x[2]))


@dataclass
class Sdf:
    """Node-grid SDF (sdf.rs:23-34): ``data`` is [nz, ny, nx], phi < 0 inside."""
    origin: tuple
    dx: float
    data: np.ndarray

    @property
    def dims(self):
        nz, ny, nx = self.data.shape
        return (nx, ny, nz)

    def bounds(self):
        nx, ny, nz = self.dims
        o = np.asarray(self.origin, dtype=np.float64)
        return o, o + np.array([(nx - 1) * self.dx, (ny - 1) * self.dx, (nz - 1) * self.dx])


def sdf_from_sinus(params: SinusParams, origin, dx: float, dims) -> Sdf:
    """Sdf::from_fn(SinusParams::implicit) evaluated on the device (scene.rs:289-297)."""
    L = _lib.load()
    nx, ny, nz = dims
    out = np.empty((nz, ny, nx))
    sp = _lib.SinusParamsC(_v3(params.semi_axes), _v3(params.center), params.taper, params.bumpiness,
                           params.socket_xz[0], params.socket_xz[1], params.socket_radius,
                           params.socket_depth, params.model_dx)
    check(L.sdr_sdf_from_sinus(C.byref(sp), _v3(origin), dx, (C.c_uint64 * 3)(nx, ny, nz), _dp(out)))
    return Sdf(tuple(origin), float(dx), out)


def sdf_from_mesh(tris: np.ndarray, dx: float, padding: float) -> Sdf:
    """Sdf::from_mesh (sdf.rs:47-86): winding-number SDF voxelised on the device."""
    L = _lib.load()
    t = np.ascontiguousarray(tris, dtype=np.float64).reshape(-1, 9)
    origin = _lib.Vec3()
    dims = (C.c_uint64 * 3)()
    check(L.sdr_sdf_mesh_grid(_dp(t), t.shape[0], dx, padding, C.byref(origin), dims))
    nx, ny, nz = (int(x) for x in dims)
    out = np.empty((nz, ny, nx))
    check(L.sdr_sdf_from_mesh(_dp(t), t.shape[0], origin, dx, dims, _dp(out)))
    return Sdf((origin.x, origin.y, origin.z), float(dx), out)


def surface_nets_volume(sdf: Sdf) -> float:
    """|signed volume| of the surface-nets mesh of a node field (sinus.rs:141-150, scene.rs:312)."""
    L = _lib.load()
    vol = C.c_double()
    nt = C.c_uint64()
    data = np.ascontiguousarray(sdf.data, dtype=np.float64)
    check(L.sdr_surface_nets_volume(_dp(data), (C.c_uint64 * 3)(*sdf.dims), _v3(sdf.origin), sdf.dx,
                                    C.byref(vol), C.byref(nt)))
    return vol.value


class Solver:
    """The fluid solver (solver.rs:143-310), device resident."""

    def __init__(self, solid: Sdf, sim_dx: float, fluid: FluidParams, needle: Needle,
                 max_particles: int = 0, device: int = -1):
        L = _lib.load()
        self.solid = solid
        self._sdf_data = np.ascontiguousarray(solid.data, dtype=np.float64)
        nx, ny, nz = solid.dims
        desc = _lib.SdfDesc(_v3(solid.origin), solid.dx, nx, ny, nz, _dp(self._sdf_data))
        self.fluid = fluid
        fp = _lib.FluidParamsC(fluid.density, _v3(fluid.gravity), fluid.flip_ratio,
                               int(fluid.particles_per_cell), fluid.volume_stiffness,
                               1 if fluid.redistribute else 0, 0, fluid.redist_cap_factor)
        self._needle = needle
        opts = _lib.SolverOptions(int(max_particles), int(device), 0)
        h = C.c_void_p()
        check(L.sdr_solver_create(C.byref(desc), sim_dx, C.byref(fp), C.byref(self._needle_c(needle)),
                                  C.byref(opts), C.byref(h)))
        self._h = h
        self._outlet = None
        self._solve = SolveParams()

    @staticmethod
    def _needle_c(n: Needle) -> _lib.NeedleC:
        return _lib.NeedleC(_v3(n.tip), _v3(n.axis), n.radius, n.flow_rate, n.inject_until)

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.load().sdr_solver_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- public fields (solver.rs:150-166)
    @property
    def outlet(self):
        return self._outlet

    @outlet.setter
    def outlet(self, box):
        self._outlet = box
        if box is None:
            check(_lib.load().sdr_solver_set_outlet(self._h, None))
        else:
            ab = _lib.Aabb(_v3(box[0]), _v3(box[1]))
            check(_lib.load().sdr_solver_set_outlet(self._h, C.byref(ab)))

    @property
    def solve(self) -> SolveParams:
        return self._solve

    @solve.setter
    def solve(self, sp: SolveParams):
        self._solve = sp
        check(_lib.load().sdr_solver_set_solve_params(self._h, C.byref(_lib.SolveParamsC(int(sp.max_iters), sp.tol))))

    @property
    def needle(self) -> Needle:
        return self._needle

    @needle.setter
    def needle(self, n: Needle):
        self._needle = n
        check(_lib.load().sdr_solver_set_needle(self._h, C.byref(self._needle_c(n))))

    def stats(self) -> _lib.SolverStats:
        st = _lib.SolverStats()
        check(_lib.load().sdr_solver_get_stats(self._h, C.byref(st)))
        return st

    def cfl(self):
        """(Solver::cfl_dt, MacGrid::max_speed) of the current state (solver.rs:262-281, grid.rs:202-206)."""
        dt, gs = C.c_double(), C.c_double()
        check(_lib.load().sdr_solver_cfl(self._h, C.byref(dt), C.byref(gs)))
        return dt.value, gs.value

    def cfl_dt(self) -> float:
        return self.cfl()[0]

    def set_candidate_capacity(self, candidates: int) -> None:
        """Entries of the redistribution candidate list (0: the particle capacity)."""
        check(_lib.load().sdr_solver_set_candidate_capacity(self._h, int(candidates)))

    def set_dot_order(self, reference_order: bool) -> None:
        """Reference dot order in the PCG (bit-exact pressure) or the faster block tree."""
        check(_lib.load().sdr_solver_set_dot_order(self._h, 1 if reference_order else 0))

    def set_pcg_kernel(self, kernel: int) -> None:
        """_lib.PCG_AUTO, PCG_ONE_BLOCK (one SM) or PCG_CLUSTER (up to 16 SMs)."""
        check(_lib.load().sdr_solver_set_pcg_kernel(self._h, int(kernel)))

    def set_pcg_ctas(self, ctas: int) -> None:
        """CTAs of the one-SM-sweep solve's cluster (0: automatic); results do not depend on it."""
        check(_lib.load().sdr_solver_set_pcg_ctas(self._h, int(ctas)))

    def set_profiling(self, on: bool, kernel_timers: bool = False) -> None:
        """Phase timing with CUDA events; kernel_timers adds the pressure-solve section timers."""
        check(_lib.load().sdr_solver_set_profiling(self._h, (2 if kernel_timers else 1) if on else 0))

    def profile(self) -> dict:
        pr = _lib.Profile()
        check(_lib.load().sdr_solver_get_profile(self._h, C.byref(pr)))
        return pr.to_dict()

    def reset_profile(self) -> None:
        check(_lib.load().sdr_solver_reset_profile(self._h))

    @property
    def time(self) -> float:
        return self.stats().time

    @property
    def steps(self) -> int:
        return self.stats().steps

    @property
    def last_pcg_iters(self) -> int:
        return self.stats().last_pcg_iters

    @property
    def last_substeps(self) -> int:
        return self.stats().last_substeps

    @property
    def drained(self) -> int:
        return self.stats().drained

    @property
    def grid_dims(self):
        st = self.stats()
        return (st.nx, st.ny, st.nz)

    @property
    def dx(self) -> float:
        return self.stats().dx

    def __len__(self) -> int:
        return int(self.stats().particles)

    # -- stepping
    def step(self, dt: float) -> None:
        check(_lib.load().sdr_solver_step(self._h, float(dt)))

    def substep(self, dt: float) -> None:
        check(_lib.load().sdr_solver_substep(self._h, float(dt)))

    def run_phase(self, phase: int, dt: float = 0.0) -> None:
        check(_lib.load().sdr_solver_run_phase(self._h, int(phase), float(dt)))

    # -- state
    def particles(self):
        n = len(self)
        pos = np.zeros((n, 3))
        vel = np.zeros((n, 3))
        got = C.c_size_t()
        check(_lib.load().sdr_solver_copy_particles(self._h, _dp(pos), _dp(vel), n, C.byref(got)))
        return pos, vel

    def particles_f32(self):
        n = len(self)
        pos = np.zeros((n, 3), dtype=np.float32)
        vel = np.zeros((n, 3), dtype=np.float32)
        got = C.c_size_t()
        fp = C.POINTER(C.c_float)
        check(_lib.load().sdr_solver_copy_particles_f32(self._h, pos.ctypes.data_as(fp), vel.ctypes.data_as(fp), n,
                                                        C.byref(got)))
        return pos, vel

    def set_particles(self, pos: np.ndarray, vel: np.ndarray) -> None:
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        vel = np.ascontiguousarray(vel, dtype=np.float64).reshape(-1, 3)
        check(_lib.load().sdr_solver_set_particles(self._h, _dp(pos), _dp(vel), pos.shape[0]))

    def set_scalars(self, time: float, emit_accum: float, steps: int, drained: int, rng: int) -> None:
        check(_lib.load().sdr_solver_set_scalars(self._h, time, emit_accum, int(steps), int(drained),
                                                 C.c_uint64(rng)))

    def ncells(self) -> int:
        nx, ny, nz = self.grid_dims
        return nx * ny * nz

    def pressure(self) -> np.ndarray:
        out = np.zeros(self.ncells())
        check(_lib.load().sdr_solver_copy_pressure(self._h, _dp(out), out.size))
        return out

    def cells(self) -> np.ndarray:
        out = np.zeros(self.ncells(), dtype=np.uint8)
        check(_lib.load().sdr_solver_copy_cells(self._h, out.ctypes.data_as(C.POINTER(C.c_uint8)), out.size))
        return out

    def cavity_mask(self) -> np.ndarray:
        out = np.zeros(self.ncells(), dtype=np.uint8)
        check(_lib.load().sdr_solver_copy_cavity_mask(self._h, out.ctypes.data_as(C.POINTER(C.c_uint8)), out.size))
        return out

    def _face_len(self, which: int) -> int:
        nx, ny, nz = self.grid_dims
        return [(nx + 1) * ny * nz, nx * (ny + 1) * nz, nx * ny * (nz + 1)][which % 3]

    def face(self, which: int) -> np.ndarray:
        out = np.zeros(self._face_len(which))
        check(_lib.load().sdr_solver_copy_face(self._h, int(which), _dp(out), out.size))
        return out

    def set_face(self, which: int, arr: np.ndarray) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
        check(_lib.load().sdr_solver_set_face(self._h, int(which), _dp(a), a.size))

    def sort(self):
        n = len(self)
        keys = np.zeros(n, dtype=np.uint32)
        perm = np.zeros(n, dtype=np.uint32)
        got = C.c_size_t()
        up = C.POINTER(C.c_uint32)
        check(_lib.load().sdr_solver_copy_sort(self._h, keys.ctypes.data_as(up), perm.ctypes.data_as(up), n,
                                               C.byref(got)))
        return keys, perm

    def _scalar(self, fn, ctype=C.c_double):
        out = ctype()
        check(fn(self._h, C.byref(out)))
        return out.value

    def max_pressure(self) -> float:
        return self._scalar(_lib.load().sdr_solver_max_pressure)

    def mean_pressure(self) -> float:
        return self._scalar(_lib.load().sdr_solver_mean_pressure)

    def max_speed(self) -> float:
        return self._scalar(_lib.load().sdr_solver_max_speed)

    def cells_fluid_count(self) -> int:
        return int(self._scalar(_lib.load().sdr_solver_cells_fluid_count, C.c_uint64))

    def max_particles_per_cell(self) -> int:
        return int(self._scalar(_lib.load().sdr_solver_max_particles_per_cell, C.c_uint64))

    # -- derived (solver.rs:225-233, 758-760)
    def particle_volume(self) -> float:
        return self.dx ** 3 / max(int(self.fluid.particles_per_cell), 1)

    def fluid_volume(self) -> float:
        return len(self) * self.particle_volume()

    def drained_volume(self) -> float:
        return self.drained * self.particle_volume()


class MetricsCollector:
    """MetricsCollector (metrics.rs:102-431): reductions run on the device."""

    def __init__(self, solver: Solver, cavity_volume: float):
        self._solver = solver
        h = C.c_void_p()
        check(_lib.load().sdr_metrics_create(solver._h, float(cavity_volume), C.byref(h)))
        self._h = h
        self.history = []

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.load().sdr_metrics_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def wall_count(self) -> int:
        out = C.c_uint64()
        check(_lib.load().sdr_metrics_wall_count(self._h, C.byref(out)))
        return out.value

    def record(self, solver: Solver, frame: int) -> dict:
        fm = _lib.FrameMetricsC()
        check(_lib.load().sdr_metrics_record(self._h, solver._h, int(frame), C.byref(fm)))
        d = fm.to_dict()
        self.history.append(d)
        return d

    def frames(self):
        return list(self.history)

    def summary(self) -> dict:
        sm = _lib.SummaryC()
        check(_lib.load().sdr_metrics_summary(self._h, C.byref(sm)))
        return sm.to_dict()

    def write_json(self, path: str) -> None:
        """metrics.json (metrics.rs:385-391), byte for byte as serde_json writes it."""
        check(_lib.load().sdr_metrics_write_json(self._h, str(path).encode()))

    def write_csv(self, path: str) -> None:
        """metrics.csv (metrics.rs:394-431), values as Rust's `{}` prints them."""
        check(_lib.load().sdr_metrics_write_csv(self._h, str(path).encode()))

    def write_summary_json(self, path: str) -> None:
        """summary.json of cmd_simulate (main.rs:306-310)."""
        sm = _lib.SummaryC()
        check(_lib.load().sdr_metrics_summary(self._h, C.byref(sm)))
        check(_lib.load().sdr_summary_write_json(C.byref(sm), str(path).encode()))


@dataclass
class BuiltScene:
    """BuiltScene (scene.rs:235-245)."""
    solver: Solver
    cavity_volume: float
    frame_dt: float
    frames: int
    resolved: ResolvedScene


def build_sdf(res: ResolvedScene, tris: Optional[np.ndarray] = None) -> Sdf:
    """The SDF of ``SceneConfig::build`` (scene.rs:279-297), voxelised on the device."""
    if res.sinus is not None:
        return sdf_from_sinus(res.sinus, res.sdf_origin, res.sdf_dx, res.sdf_dims)
    if tris is None:
        tris = load_mesh(res.mesh_path) * MM
    return sdf_from_mesh(tris, res.sdf_dx, res.mesh_padding)


def cavity_volume(res: ResolvedScene, sdf: Sdf, tris: Optional[np.ndarray] = None) -> float:
    """``cavity_mesh.signed_volume().abs()`` (scene.rs:312)."""
    if res.sinus is not None:
        # The surface-nets grid of SinusParams::generate is the SDF grid itself.
        return surface_nets_volume(sdf)
    if tris is None:
        tris = load_mesh(res.mesh_path) * MM
    t = np.asarray(tris, dtype=np.float64).reshape(-1, 3, 3)
    a, b, c = t[:, 0], t[:, 1], t[:, 2]
    cr = np.cross(b, c)
    terms = (a[:, 0] * cr[:, 0] + a[:, 1] * cr[:, 1] + a[:, 2] * cr[:, 2]) / 6.0
    return abs(float(np.cumsum(terms)[-1])) if len(terms) else 0.0  # sequential sum, mesh.rs:63-70


def build_scene(cfg: SceneConfig, sdf: Optional[Sdf] = None, max_particles: int = 0) -> BuiltScene:
    """SceneConfig::build (scene.rs:266-334) on the device."""
    res = cfg.resolve()
    tris = None
    if res.sinus is None:
        tris = load_mesh(res.mesh_path) * MM
    sdf = sdf if sdf is not None else build_sdf(res, tris)
    vol = cavity_volume(res, sdf, tris)
    s = Solver(sdf, res.sim_dx, res.fluid, res.needle, max_particles=max_particles)
    s.solve = res.solve
    s.outlet = res.outlet
    return BuiltScene(solver=s, cavity_volume=vol, frame_dt=res.frame_dt, frames=res.frames, resolved=res)
