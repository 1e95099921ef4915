"""ctypes bindings of the CPU oracle (sdr_oracle.cpp).

TEST INFRASTRUCTURE ONLY: the oracle is the checker for the CUDA path. Only
tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this
package; the product (``sdr_b200``) never does.

The oracle restates uselessgoddess/sdr's ``src/solver.rs``, ``src/pressure.rs``,
``src/grid.rs``, ``src/sdf.rs``, ``src/sinus.rs``, ``src/surface_nets.rs`` and
``src/metrics.rs`` in C++ f64 with the reference's operation order. Parity
pins: the reference's own known-answer tests (tests/test_oracle_*.py).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

PHASE_EMIT, PHASE_CLASSIFY, PHASE_P2G, PHASE_SAVE_GRID, PHASE_ADD_FORCES = 0, 1, 2, 3, 4
PHASE_PROJECT, PHASE_EXTRAPOLATE, PHASE_G2P, PHASE_ADVECT, PHASE_BOUNDS = 5, 6, 7, 8, 9
PHASE_REDISTRIBUTE, PHASE_CLOCK = 10, 11
SOLID, FLUID, AIR = 0, 1, 2


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile (gcc, f64, no FMA)."""
    src = os.path.join(_HERE, "sdr_oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return _LIB_PATH


class OrcFluid(C.Structure):
    _fields_ = [("density", C.c_double), ("gravity", C.c_double * 3), ("flip_ratio", C.c_double),
                ("particles_per_cell", C.c_uint64), ("volume_stiffness", C.c_double),
                ("redistribute", C.c_int32), ("_pad", C.c_int32), ("redist_cap_factor", C.c_double)]


class OrcNeedle(C.Structure):
    _fields_ = [("tip", C.c_double * 3), ("axis", C.c_double * 3), ("radius", C.c_double),
                ("flow_rate", C.c_double), ("inject_until", C.c_double)]


class OrcSinus(C.Structure):
    _fields_ = [("semi_axes", C.c_double * 3), ("center", C.c_double * 3), ("taper", C.c_double),
                ("bumpiness", C.c_double), ("socket_xz", C.c_double * 2),
                ("socket_radius", C.c_double), ("socket_depth", C.c_double),
                ("model_dx", C.c_double)]


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


class OrcSlicePlane(C.Structure):  # render.rs:45-56
    _fields_ = [("hax", C.c_int32), ("vax", C.c_int32), ("oax", C.c_int32), ("flip_v", C.c_int32),
                ("project", C.c_int32), ("amber", C.c_int32), ("slice", C.c_double), ("slab", C.c_double)]


class OrcFrameMetrics(C.Structure):
    _fields_ = _fields(_FM)

    def to_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class OrcSummary(C.Structure):
    _fields_ = _fields(_SM)

    def to_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        _declare(_lib)
    return _lib


def _declare(L):
    d, u64, i32, vp = C.c_double, C.c_uint64, C.c_int, C.c_void_p
    P = C.POINTER
    sig = {
        "orc_set_threads": (None, [i32]),
        "orc_get_threads": (i32, []),
        "orc_point_triangle_distance_sq": (d, [P(d)] * 4),
        "orc_signed_distance_to_mesh": (d, [P(d), P(d), C.c_size_t]),
        "orc_sdf_mesh_grid": (None, [P(d), C.c_size_t, d, d, P(d), P(u64)]),
        "orc_sdf_from_mesh": (None, [P(d), C.c_size_t, P(d), d, P(u64), P(d)]),
        "orc_sinus_implicit": (d, [P(OrcSinus), P(d)]),
        "orc_sinus_bounds": (None, [P(OrcSinus), P(d), P(d)]),
        "orc_sinus_socket_bottom_y": (d, [P(OrcSinus)]),
        "orc_sinus_suggested_needle": (None, [P(OrcSinus), P(d), P(d)]),
        "orc_sdf_from_sinus": (None, [P(OrcSinus), P(d), d, P(u64), P(d)]),
        "orc_sinus_mesh_volume": (d, [P(OrcSinus), P(u64)]),
        "orc_sinus_mesh": (C.c_size_t, [P(OrcSinus), P(d), C.c_size_t]),
        "orc_mesh_signed_volume": (d, [P(d), C.c_size_t]),
        "orc_sdf_sample": (d, [P(d), P(u64), P(d), d, P(d)]),
        "orc_sdf_gradient": (None, [P(d), P(u64), P(d), d, P(d), P(d)]),
        "orc_solver_new": (vp, [P(d), P(u64), P(d), d, d, P(OrcFluid), P(OrcNeedle)]),
        "orc_solver_free": (None, [vp]),
        "orc_solver_set_outlet": (None, [vp, i32, P(d), P(d)]),
        "orc_solver_set_solve": (None, [vp, u64, d]),
        "orc_solver_set_needle": (None, [vp, P(OrcNeedle)]),
        "orc_solver_step": (None, [vp, d]),
        "orc_solver_substep": (None, [vp, d]),
        "orc_solver_phase": (None, [vp, i32, d]),
        "orc_solver_cfl_dt": (d, [vp]),
        "orc_solver_grid": (None, [vp, P(u64), P(d), P(d)]),
        "orc_solver_num_particles": (C.c_size_t, [vp]),
        "orc_solver_get_particles": (None, [vp, P(d), P(d)]),
        "orc_solver_set_particles": (None, [vp, C.c_size_t, P(d), P(d)]),
        "orc_solver_get_scalars": (None, [vp, P(d), P(d), P(u64), P(u64), P(u64), P(u64), P(u64)]),
        "orc_solver_set_scalars": (None, [vp, d, d, u64, u64, u64]),
        "orc_solver_get_face": (None, [vp, i32, P(d)]),
        "orc_solver_set_face": (None, [vp, i32, P(d)]),
        "orc_solver_get_cells": (None, [vp, P(C.c_uint8)]),
        "orc_solver_set_cells": (None, [vp, P(C.c_uint8)]),
        "orc_solver_get_cavity_mask": (None, [vp, P(C.c_uint8)]),
        "orc_solver_get_pressure": (None, [vp, P(d)]),
        "orc_solver_get_source": (None, [vp, d, P(d)]),
        "orc_solver_max_pressure": (d, [vp]),
        "orc_solver_mean_pressure": (d, [vp]),
        "orc_solver_max_speed": (d, [vp]),
        "orc_solver_kinetic_energy": (d, [vp]),
        "orc_solver_max_particles_per_cell": (u64, [vp]),
        "orc_solver_cells_fluid_count": (u64, [vp]),
        "orc_solver_grid_max_speed": (d, [vp]),
        "orc_solver_phase_times": (None, [vp, P(d)]),
        "orc_project": (u64, [u64, u64, u64, d, P(d), P(d), P(d), P(C.c_uint8), d, d, u64, d,
                              P(d), P(d), P(d)]),
        "orc_build_mic0": (None, [u64, u64, u64, P(C.c_uint8), P(d)]),
        "orc_apply_mic0": (None, [u64, u64, u64, P(C.c_uint8), P(d), P(d), P(d)]),
        "orc_dot": (d, [P(d), P(d), C.c_size_t]),
        "orc_metrics_new": (vp, [vp, d]),
        "orc_metrics_free": (None, [vp]),
        "orc_metrics_record": (None, [vp, vp, u64, P(OrcFrameMetrics)]),
        "orc_metrics_summary": (None, [vp, P(OrcSummary)]),
        "orc_metrics_wall_count": (u64, [vp]),
        "orc_metrics_get_masks": (None, [vp, P(C.c_uint8), P(C.c_uint8)]),
        "orc_membrane_stats": (None, [P(d), C.c_size_t, d, P(d), P(d), P(u64)]),
        "orc_hash_jitter": (None, [u64, P(d)]),
        "orc_render_slice_dims": (None, [vp, P(OrcSlicePlane), C.c_uint32, P(C.c_uint32), P(C.c_uint32)]),
        "orc_render_slice": (None, [vp, P(OrcSlicePlane), C.c_uint32, d, P(C.c_uint8)]),
        "orc_render_timeseries": (None, [P(OrcFrameMetrics), C.c_size_t, C.c_uint32, C.c_uint32, P(C.c_uint8)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _u8p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


def _u64p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint64))


def _vec(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


# ---------------------------------------------------------------- geometry
def point_triangle_distance_sq(p, a, b, c) -> float:
    return lib().orc_point_triangle_distance_sq(*(_dp(_vec(x)) for x in (p, a, b, c)))


def signed_distance_to_mesh(p, tris: np.ndarray) -> float:
    t = np.ascontiguousarray(tris, dtype=np.float64).reshape(-1, 9)
    return lib().orc_signed_distance_to_mesh(_dp(_vec(p)), _dp(t), t.shape[0])


@dataclass
class SdfGrid:
    """A node-grid SDF (sdf.rs:23-34); data is [nz, ny, nx] x-fastest."""
    origin: np.ndarray
    dx: float
    data: np.ndarray

    @property
    def dims(self):
        nz, ny, nx = self.data.shape
        return (nx, ny, nz)

    def _dims_arr(self):
        return np.array(self.dims, dtype=np.uint64)

    def sample(self, p) -> float:
        return lib().orc_sdf_sample(_dp(self.data), _u64p(self._dims_arr()), _dp(_vec(self.origin)),
                                    self.dx, _dp(_vec(p)))

    def gradient(self, p) -> np.ndarray:
        g = np.zeros(3)
        lib().orc_sdf_gradient(_dp(self.data), _u64p(self._dims_arr()), _dp(_vec(self.origin)),
                               self.dx, _dp(_vec(p)), _dp(g))
        return g

    def bounds(self):
        nx, ny, nz = self.dims
        o = np.asarray(self.origin, dtype=np.float64)
        return o, o + np.array([(nx - 1) * self.dx, (ny - 1) * self.dx, (nz - 1) * self.dx])


def sdf_from_fn(origin, dx: float, dims, f) -> SdfGrid:
    """Sdf::from_fn (sdf.rs:90-116) with a Python callable (small grids only)."""
    nx, ny, nz = dims
    data = np.empty((nz, ny, nx))
    o = np.asarray(origin, dtype=np.float64)
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                data[k, j, i] = f(np.array([o[0] + i * dx, o[1] + j * dx, o[2] + k * dx]))
    return SdfGrid(o.copy(), float(dx), data)


def sdf_mesh_grid(tris: np.ndarray, dx: float, padding: float):
    t = np.ascontiguousarray(tris, dtype=np.float64).reshape(-1, 9)
    origin = np.zeros(3)
    dims = np.zeros(3, dtype=np.uint64)
    lib().orc_sdf_mesh_grid(_dp(t), t.shape[0], dx, padding, _dp(origin), _u64p(dims))
    return origin, tuple(int(x) for x in dims)


def sdf_from_mesh(tris: np.ndarray, dx: float, padding: float) -> SdfGrid:
    """Sdf::from_mesh (sdf.rs:47-86): winding-number sign, closest-point distance."""
    t = np.ascontiguousarray(tris, dtype=np.float64).reshape(-1, 9)
    origin, dims = sdf_mesh_grid(t, dx, padding)
    data = np.empty((dims[2], dims[1], dims[0]))
    lib().orc_sdf_from_mesh(_dp(t), t.shape[0], _dp(origin), dx, _u64p(np.array(dims, dtype=np.uint64)),
                            _dp(data))
    return SdfGrid(origin, float(dx), data)


def sinus_struct(p) -> OrcSinus:
    s = OrcSinus()
    s.semi_axes[:] = list(p.semi_axes)
    s.center[:] = list(p.center)
    s.taper = p.taper
    s.bumpiness = p.bumpiness
    s.socket_xz[:] = list(p.socket_xz)
    s.socket_radius = p.socket_radius
    s.socket_depth = p.socket_depth
    s.model_dx = p.model_dx
    return s


def sinus_implicit(params, p) -> float:
    return lib().orc_sinus_implicit(C.byref(sinus_struct(params)), _dp(_vec(p)))


def sinus_bounds(params):
    mn, mx = np.zeros(3), np.zeros(3)
    lib().orc_sinus_bounds(C.byref(sinus_struct(params)), _dp(mn), _dp(mx))
    return mn, mx


def sinus_socket_bottom_y(params) -> float:
    return lib().orc_sinus_socket_bottom_y(C.byref(sinus_struct(params)))


def sinus_suggested_needle(params):
    tip, axis = np.zeros(3), np.zeros(3)
    lib().orc_sinus_suggested_needle(C.byref(sinus_struct(params)), _dp(tip), _dp(axis))
    return tip, axis


def sdf_from_sinus(params, origin, dx: float, dims) -> SdfGrid:
    nx, ny, nz = dims
    data = np.empty((nz, ny, nx))
    o = _vec(origin)
    lib().orc_sdf_from_sinus(C.byref(sinus_struct(params)), _dp(o), dx,
                             _u64p(np.array(dims, dtype=np.uint64)), _dp(data))
    return SdfGrid(o.copy(), float(dx), data)


def sinus_mesh_volume(params):
    nt = C.c_uint64(0)
    v = lib().orc_sinus_mesh_volume(C.byref(sinus_struct(params)), C.byref(nt))
    return v, int(nt.value)


def sinus_mesh(params) -> np.ndarray:
    s = sinus_struct(params)
    nt = lib().orc_sinus_mesh(C.byref(s), None, 0)
    out = np.empty((nt, 9))
    lib().orc_sinus_mesh(C.byref(s), _dp(out), nt)
    return out


def mesh_signed_volume(tris: np.ndarray) -> float:
    t = np.ascontiguousarray(tris, dtype=np.float64).reshape(-1, 9)
    return lib().orc_mesh_signed_volume(_dp(t), t.shape[0])


def hash_jitter(key: int) -> np.ndarray:
    out = np.zeros(3)
    lib().orc_hash_jitter(C.c_uint64(key), _dp(out))
    return out


def membrane_stats(values: Sequence[float], cap: float):
    v = _vec(values) if len(values) else np.zeros(1)
    mean, peak, art = C.c_double(), C.c_double(), C.c_uint64()
    lib().orc_membrane_stats(_dp(v), len(values), cap, C.byref(mean), C.byref(peak), C.byref(art))
    return mean.value, peak.value, int(art.value)


def dot(a: np.ndarray, b: np.ndarray) -> float:
    a = _vec(a)
    b = _vec(b)
    return lib().orc_dot(_dp(a), _dp(b), a.size)


def project(nx, ny, nz, dx, u, v, w, cells, rho, dt, max_iters, tol, source=None):
    """project_capturing_with_source (pressure.rs:123-239) on numpy arrays.

    Returns (u, v, w, pressure, iters, residual)."""
    u, v, w = _vec(u).copy(), _vec(v).copy(), _vec(w).copy()
    cells = np.ascontiguousarray(cells, dtype=np.uint8).reshape(-1)
    p = np.zeros(nx * ny * nz)
    res = C.c_double()
    src = None if source is None else _dp(_vec(source))
    iters = lib().orc_project(nx, ny, nz, dx, _dp(u), _dp(v), _dp(w), _u8p(cells), rho, dt,
                              max_iters, tol, src, _dp(p), C.byref(res))
    return u, v, w, p, int(iters), res.value


def build_mic0(nx, ny, nz, cells) -> np.ndarray:
    cells = np.ascontiguousarray(cells, dtype=np.uint8).reshape(-1)
    out = np.zeros(nx * ny * nz)
    lib().orc_build_mic0(nx, ny, nz, _u8p(cells), _dp(out))
    return out


def apply_mic0(nx, ny, nz, cells, precon, r) -> np.ndarray:
    cells = np.ascontiguousarray(cells, dtype=np.uint8).reshape(-1)
    z = np.zeros(nx * ny * nz)
    lib().orc_apply_mic0(nx, ny, nz, _u8p(cells), _dp(_vec(precon)), _dp(_vec(r)), _dp(z))
    return z


# ---------------------------------------------------------------- solver
@dataclass
class Fluid:
    """FluidParams (solver.rs:41-85) with the reference defaults."""
    density: float = 1000.0
    gravity: Sequence[float] = (0.0, -9.81, 0.0)
    flip_ratio: float = 0.95
    particles_per_cell: int = 8
    volume_stiffness: float = 1.0
    redistribute: bool = True
    redist_cap_factor: float = 1.0

    def to_c(self) -> OrcFluid:
        f = OrcFluid()
        f.density = self.density
        f.gravity[:] = list(self.gravity)
        f.flip_ratio = self.flip_ratio
        f.particles_per_cell = int(self.particles_per_cell)
        f.volume_stiffness = self.volume_stiffness
        f.redistribute = 1 if self.redistribute else 0
        f.redist_cap_factor = self.redist_cap_factor
        return f


@dataclass
class Needle:
    """Needle (solver.rs:89-115)."""
    tip: Sequence[float]
    axis: Sequence[float]
    radius: float
    flow_rate: float
    inject_until: float = float("inf")

    def to_c(self) -> OrcNeedle:
        n = OrcNeedle()
        n.tip[:] = list(self.tip)
        n.axis[:] = list(self.axis)
        n.radius = self.radius
        n.flow_rate = self.flow_rate
        n.inject_until = self.inject_until
        return n


class Solver:
    """The oracle's Solver (solver.rs:143-310)."""

    def __init__(self, sdf: SdfGrid, sim_dx: float, fluid: Fluid, needle: Needle):
        self._sdf_data = np.ascontiguousarray(sdf.data, dtype=np.float64)
        dims = np.array(sdf.dims, dtype=np.uint64)
        self.sdf = sdf
        self.fluid = fluid
        self._needle = needle
        self._h = lib().orc_solver_new(_dp(self._sdf_data), _u64p(dims), _dp(_vec(sdf.origin)),
                                       sdf.dx, sim_dx, C.byref(fluid.to_c()), C.byref(needle.to_c()))
        self.outlet = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.orc_solver_free(h)
            self._h = None

    # configuration
    def set_outlet(self, outlet):
        self.outlet = outlet
        if outlet is None:
            lib().orc_solver_set_outlet(self._h, 0, None, None)
        else:
            lib().orc_solver_set_outlet(self._h, 1, _dp(_vec(outlet[0])), _dp(_vec(outlet[1])))

    def set_solve(self, max_iters: int, tol: float):
        lib().orc_solver_set_solve(self._h, int(max_iters), float(tol))

    @property
    def needle(self) -> Needle:
        return self._needle

    def set_needle(self, needle: Needle):
        self._needle = needle
        lib().orc_solver_set_needle(self._h, C.byref(needle.to_c()))

    # stepping
    def step(self, dt: float):
        lib().orc_solver_step(self._h, dt)

    def substep(self, dt: float):
        lib().orc_solver_substep(self._h, dt)

    def phase(self, phase: int, dt: float = 0.0):
        lib().orc_solver_phase(self._h, phase, dt)

    def cfl_dt(self) -> float:
        return lib().orc_solver_cfl_dt(self._h)

    # state
    @property
    def grid(self):
        dims = np.zeros(3, dtype=np.uint64)
        origin = np.zeros(3)
        dx = C.c_double()
        lib().orc_solver_grid(self._h, _u64p(dims), _dp(origin), C.byref(dx))
        return tuple(int(x) for x in dims), origin, dx.value

    def __len__(self):
        return lib().orc_solver_num_particles(self._h)

    def particles(self):
        n = len(self)
        pos = np.zeros((n, 3))
        vel = np.zeros((n, 3))
        if n:
            lib().orc_solver_get_particles(self._h, _dp(pos), _dp(vel))
        return pos, vel

    def set_particles(self, pos: np.ndarray, vel: np.ndarray):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        vel = np.ascontiguousarray(vel, dtype=np.float64).reshape(-1, 3)
        lib().orc_solver_set_particles(self._h, pos.shape[0], _dp(pos), _dp(vel))

    def scalars(self) -> dict:
        t, ea = C.c_double(), C.c_double()
        st, it, sub, dr, rng = (C.c_uint64() for _ in range(5))
        lib().orc_solver_get_scalars(self._h, C.byref(t), C.byref(ea), C.byref(st), C.byref(it),
                                     C.byref(sub), C.byref(dr), C.byref(rng))
        return dict(time=t.value, emit_accum=ea.value, steps=st.value, last_pcg_iters=it.value,
                    last_substeps=sub.value, drained=dr.value, rng=rng.value)

    def set_scalars(self, time: float, emit_accum: float, steps: int, drained: int, rng: int):
        lib().orc_solver_set_scalars(self._h, time, emit_accum, steps, drained, C.c_uint64(rng))

    def _face_len(self, which: int) -> int:
        (nx, ny, nz), _, _ = self.grid
        return [(nx + 1) * ny * nz, nx * (ny + 1) * nz, nx * ny * (nz + 1)][which % 3]

    def face(self, which: int) -> np.ndarray:
        out = np.zeros(self._face_len(which))
        lib().orc_solver_get_face(self._h, which, _dp(out))
        return out

    def set_face(self, which: int, arr: np.ndarray):
        a = _vec(arr)
        assert a.size == self._face_len(which)
        lib().orc_solver_set_face(self._h, which, _dp(a))

    def ncells(self) -> int:
        (nx, ny, nz), _, _ = self.grid
        return nx * ny * nz

    def cells(self) -> np.ndarray:
        out = np.zeros(self.ncells(), dtype=np.uint8)
        lib().orc_solver_get_cells(self._h, _u8p(out))
        return out

    def set_cells(self, cells: np.ndarray):
        c = np.ascontiguousarray(cells, dtype=np.uint8).reshape(-1)
        lib().orc_solver_set_cells(self._h, _u8p(c))

    def cavity_mask(self) -> np.ndarray:
        out = np.zeros(self.ncells(), dtype=np.uint8)
        lib().orc_solver_get_cavity_mask(self._h, _u8p(out))
        return out

    def pressure(self) -> np.ndarray:
        out = np.zeros(self.ncells())
        lib().orc_solver_get_pressure(self._h, _dp(out))
        return out

    def source(self, dt: float) -> np.ndarray:
        out = np.zeros(self.ncells())
        lib().orc_solver_get_source(self._h, dt, _dp(out))
        return out

    def max_pressure(self): return lib().orc_solver_max_pressure(self._h)
    def mean_pressure(self): return lib().orc_solver_mean_pressure(self._h)
    def max_speed(self): return lib().orc_solver_max_speed(self._h)

    def render_slice(self, plane: dict, target_px: int, vmax: float = 0.0) -> np.ndarray:
        """render_slice (render.rs:139-236) as an (h, w, 3) uint8 image; plane has the
        SlicePlane fields (hax, vax, oax, slice, slab, flip_v, project, amber)."""
        pl = OrcSlicePlane(**{k: plane[k] for k, _ in OrcSlicePlane._fields_})
        w, h = C.c_uint32(), C.c_uint32()
        lib().orc_render_slice_dims(self._h, C.byref(pl), int(target_px), C.byref(w), C.byref(h))
        img = np.zeros((h.value, w.value, 3), dtype=np.uint8)
        lib().orc_render_slice(self._h, C.byref(pl), int(target_px), float(vmax),
                               img.ctypes.data_as(C.POINTER(C.c_uint8)))
        return img
    def kinetic_energy(self): return lib().orc_solver_kinetic_energy(self._h)
    def max_particles_per_cell(self): return int(lib().orc_solver_max_particles_per_cell(self._h))
    def cells_fluid_count(self): return int(lib().orc_solver_cells_fluid_count(self._h))
    def grid_max_speed(self): return lib().orc_solver_grid_max_speed(self._h)

    def phase_times(self) -> np.ndarray:
        out = np.zeros(12)
        lib().orc_solver_phase_times(self._h, _dp(out))
        return out

    def particle_volume(self) -> float:
        _, _, dx = self.grid
        return dx ** 3 / max(self.fluid.particles_per_cell, 1)


class Metrics:
    """MetricsCollector (metrics.rs:102-446)."""

    def __init__(self, solver: Solver, cavity_volume: float):
        self._solver = solver
        self._h = lib().orc_metrics_new(solver._h, cavity_volume)
        self.frames = []

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.orc_metrics_free(h)
            self._h = None

    def record(self, solver: Solver, frame: int) -> dict:
        out = OrcFrameMetrics()
        lib().orc_metrics_record(self._h, solver._h, frame, C.byref(out))
        d = out.to_dict()
        self.frames.append(d)
        return d

    def summary(self) -> dict:
        out = OrcSummary()
        lib().orc_metrics_summary(self._h, C.byref(out))
        return out.to_dict()

    @property
    def wall_count(self) -> int:
        return int(lib().orc_metrics_wall_count(self._h))

    def masks(self):
        n = self._solver.ncells()
        a = np.zeros(n, dtype=np.uint8)
        b = np.zeros(n, dtype=np.uint8)
        lib().orc_metrics_get_masks(self._h, _u8p(a), _u8p(b))
        return a, b


def render_timeseries(frames, width: int, height: int) -> np.ndarray:
    """render_timeseries (render.rs:351-406): frames are FrameMetrics dicts."""
    arr = (OrcFrameMetrics * max(len(frames), 1))()
    for i, f in enumerate(frames):
        for k, _ in OrcFrameMetrics._fields_:
            setattr(arr[i], k, f[k])
    img = np.zeros((height, width, 3), dtype=np.uint8)
    lib().orc_render_timeseries(arr, len(frames), int(width), int(height), img.ctypes.data_as(C.POINTER(C.c_uint8)))
    return img
