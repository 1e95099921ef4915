"""Doctor-facing scene configuration (clinical units) -> SI solver inputs.

Mirrors uselessgoddess/sdr ``src/scene.rs`` (TOML schema, defaults, unit
conversion, needle resolution, derived outlet) and the parametric cavity of
``src/sinus.rs`` (bounds, socket, suggested needle). Unknown keys are rejected
like ``#[serde(deny_unknown_fields)]`` (scene.rs:27).

Float arithmetic here is IEEE f64 in the reference's operation order, so a
resolved scene carries bit-identical numbers to the reference's ``build()``.
The GPU-side work (SDF voxelisation, solver creation) lives in
:mod:`sdr_b200.solver`; this module is pure configuration.
"""
from __future__ import annotations

import copy
import math
import os
import tomllib
from dataclasses import dataclass, field
from typing import Optional, Tuple

MM = 1e-3          # scene.rs:22
ML_PER_S = 1e-6    # scene.rs:23

Vec3 = Tuple[float, float, float]


class SceneError(ValueError):
    """Invalid scene configuration (the reference's ``anyhow::bail!`` in scene.rs)."""


@dataclass
class SinusParams:
    """Parametric cavity, SI units (sinus.rs:26-62)."""
    semi_axes: Vec3 = (0.017, 0.016, 0.013)
    center: Vec3 = (0.0, 0.0, 0.0)
    taper: float = 0.6
    bumpiness: float = 0.12
    socket_xz: Tuple[float, float] = (0.006, 0.0)
    socket_radius: float = 0.0025
    socket_depth: float = 0.006
    model_dx: float = 0.0007

    def socket_bottom_y(self) -> float:  # sinus.rs:77-79
        return self.center[1] - self.semi_axes[1] - self.socket_depth

    def socket_top_y(self) -> float:  # sinus.rs:83-85
        return self.center[1] - 0.5 * self.semi_axes[1]

    def bounds(self):  # sinus.rs:122-138
        f = 1.0 + self.bumpiness
        a = tuple(x * f for x in self.semi_axes)
        mn = [self.center[i] - a[i] for i in range(3)]
        mx = [self.center[i] + a[i] for i in range(3)]
        sx, sz = self.socket_xz
        yb = self.socket_bottom_y()
        for p in ((sx + self.socket_radius, yb, sz + self.socket_radius),
                  (sx - self.socket_radius, yb, sz - self.socket_radius)):
            for i in range(3):
                mn[i] = min(mn[i], p[i])
                mx[i] = max(mx[i], p[i])
        pad = 2.0 * self.model_dx
        return tuple(x - pad for x in mn), tuple(x + pad for x in mx)

    def suggested_needle(self):  # sinus.rs:154-160
        sx, sz = self.socket_xz
        tip = (sx, self.socket_top_y() + self.semi_axes[1] * 0.15, sz)
        return tip, (0.0, 1.0, 0.0)


@dataclass
class FluidParams:
    """FluidParams (solver.rs:41-85)."""
    density: float = 1000.0
    gravity: Vec3 = (0.0, -9.81, 0.0)
    flip_ratio: float = 0.95
    particles_per_cell: int = 8
    volume_stiffness: float = 1.0
    redistribute: bool = True
    redist_cap_factor: float = 1.0


@dataclass
class Needle:
    """Needle (solver.rs:89-115)."""
    tip: Vec3
    axis: Vec3
    radius: float
    flow_rate: float
    inject_until: float = math.inf

    def jet_speed(self) -> float:  # solver.rs:107-114
        area = math.pi * self.radius * self.radius
        return self.flow_rate / area if area > 0.0 else 0.0


@dataclass
class SolveParams:
    """SolveParams (pressure.rs:36-50)."""
    max_iters: int = 200
    tol: float = 1e-6


def _sinus_defaults():
    p = SinusParams()
    return dict(
        mesh=None,
        semi_axes_mm=[p.semi_axes[0] / MM, p.semi_axes[1] / MM, p.semi_axes[2] / MM],
        center_mm=[p.center[0] / MM, p.center[1] / MM, p.center[2] / MM],
        taper=p.taper,
        bumpiness=p.bumpiness,
        socket_xz_mm=[p.socket_xz[0] / MM, p.socket_xz[1] / MM],
        socket_radius_mm=p.socket_radius / MM,
        socket_depth_mm=p.socket_depth / MM,
        model_resolution_mm=p.model_dx / MM,
    )


def _fluid_defaults():
    f = FluidParams()
    return dict(density_kg_m3=f.density, gravity_m_s2=list(f.gravity), flip_ratio=f.flip_ratio,
                particles_per_cell=f.particles_per_cell, volume_stiffness=f.volume_stiffness,
                redistribute=f.redistribute, redist_cap_factor=f.redist_cap_factor)


_DEFAULTS = {  # scene.rs:63-215
    "sinus": _sinus_defaults,
    "needle": lambda: dict(tip_mm=None, auto=True, axis=[0.0, 1.0, 0.0], diameter_mm=0.8,
                           flow_rate_ml_s=5.0, inject_s=None),
    "fluid": _fluid_defaults,
    "sim": lambda: dict(resolution_mm=1.0, duration_s=2.0, frames=60, pcg_iters=200, pcg_tol=1e-6),
}
_INT_KEYS = {("fluid", "particles_per_cell"), ("sim", "frames"), ("sim", "pcg_iters")}


@dataclass
class ResolvedScene:
    """Everything ``SceneConfig::build`` derives (scene.rs:266-334), minus the SDF data."""
    sim_dx: float
    fluid: FluidParams
    needle: Needle
    outlet: Optional[Tuple[Vec3, Vec3]]
    solve: SolveParams
    frames: int
    frame_dt: float
    # geometry: parametric or mesh
    sinus: Optional[SinusParams]
    mesh_path: Optional[str]
    # SDF grid (origin, dx, dims) for the parametric path; mesh grids depend on the mesh bounds.
    sdf_origin: Optional[Vec3] = None
    sdf_dx: float = 0.0
    sdf_dims: Optional[Tuple[int, int, int]] = None
    mesh_padding: float = 0.0


class SceneConfig:
    """Top-level scene (scene.rs:28-36), parsed from TOML in clinical units."""

    def __init__(self, data: Optional[dict] = None):
        data = copy.deepcopy(data or {})
        unknown = set(data) - {"sinus", "needle", "fluid", "sim", "outlet"}
        if unknown:
            raise SceneError(f"unknown field(s) {sorted(unknown)} in scene")
        for sec, mk in _DEFAULTS.items():
            d = mk()
            given = data.get(sec, {})
            if not isinstance(given, dict):
                raise SceneError(f"[{sec}] must be a table")
            bad = set(given) - set(d)
            if bad:
                raise SceneError(f"unknown field(s) {sorted(bad)} in [{sec}]")
            for k, v in given.items():
                if (sec, k) in _INT_KEYS:
                    if isinstance(v, bool) or not isinstance(v, int) or v < 0:
                        raise SceneError(f"[{sec}].{k} must be a non-negative integer")
                elif isinstance(d[k], bool):
                    if not isinstance(v, bool):
                        raise SceneError(f"[{sec}].{k} must be a boolean")
                elif isinstance(d[k], float) and not isinstance(v, bool) and isinstance(v, (int, float)):
                    v = float(v)
                elif isinstance(d[k], list) or k in ("tip_mm",):
                    v = [float(x) for x in v]
                d[k] = v
            setattr(self, sec, d)
        self.outlet = None
        if data.get("outlet") is not None:
            o = data["outlet"]
            if set(o) != {"min_mm", "max_mm"}:
                raise SceneError("[outlet] needs exactly min_mm and max_mm")
            self.outlet = {"min_mm": [float(x) for x in o["min_mm"]],
                           "max_mm": [float(x) for x in o["max_mm"]]}
        self.base_dir = "."

    @classmethod
    def from_toml_str(cls, s: str) -> "SceneConfig":
        try:
            return cls(tomllib.loads(s))
        except tomllib.TOMLDecodeError as e:
            raise SceneError(f"parsing scene TOML: {e}") from e

    @classmethod
    def from_toml_file(cls, path: str) -> "SceneConfig":
        with open(path, "rb") as f:
            text = f.read().decode()
        cfg = cls.from_toml_str(text)
        cfg.base_dir = os.path.dirname(os.path.abspath(path))
        return cfg

    # -- conversions (scene.rs:80-98, 171-187)
    def sinus_params(self) -> SinusParams:
        s = self.sinus
        return SinusParams(
            semi_axes=tuple(x * MM for x in s["semi_axes_mm"]),
            center=tuple(x * MM for x in s["center_mm"]),
            taper=s["taper"], bumpiness=s["bumpiness"],
            socket_xz=(s["socket_xz_mm"][0] * MM, s["socket_xz_mm"][1] * MM),
            socket_radius=s["socket_radius_mm"] * MM,
            socket_depth=s["socket_depth_mm"] * MM,
            model_dx=s["model_resolution_mm"] * MM,
        )

    def fluid_params(self) -> FluidParams:
        f = self.fluid
        return FluidParams(density=f["density_kg_m3"], gravity=tuple(f["gravity_m_s2"]),
                           flip_ratio=f["flip_ratio"], particles_per_cell=f["particles_per_cell"],
                           volume_stiffness=f["volume_stiffness"], redistribute=f["redistribute"],
                           redist_cap_factor=f["redist_cap_factor"])

    def resolve_needle(self, auto) -> Needle:  # scene.rs:336-373
        n = self.needle
        radius = 0.5 * n["diameter_mm"] * MM
        if radius <= 0.0:
            raise SceneError("needle.diameter_mm must be positive")
        flow_rate = n["flow_rate_ml_s"] * ML_PER_S
        if n["tip_mm"] is not None:
            tip = tuple(x * MM for x in n["tip_mm"])
            axis = tuple(n["axis"])
        elif n["auto"]:
            if auto is None:
                raise SceneError("needle.auto is set but the sinus is a loaded mesh; specify needle.tip_mm")
            tip, axis = auto
        else:
            raise SceneError("set either needle.tip_mm or needle.auto = true")
        ln = math.sqrt(axis[0] * axis[0] + axis[1] * axis[1] + axis[2] * axis[2])
        axis = tuple(a / ln for a in axis) if ln > 1e-12 else (0.0, 0.0, 0.0)
        if math.sqrt(sum(a * a for a in axis)) < 0.5:
            raise SceneError("needle.axis must be a non-zero direction")
        inject = n["inject_s"]
        return Needle(tip=tip, axis=axis, radius=radius, flow_rate=flow_rate,
                      inject_until=math.inf if inject is None else float(inject))

    def resolve(self) -> ResolvedScene:  # scene.rs:266-334 without the SDF voxelisation
        if self.sim["resolution_mm"] <= 0.0:
            raise SceneError("sim.resolution_mm must be positive")
        if self.fluid["flip_ratio"] < 0.0 or self.fluid["flip_ratio"] > 1.0:
            raise SceneError("fluid.flip_ratio must be in [0, 1]")
        sim_dx = self.sim["resolution_mm"] * MM
        fluid = self.fluid_params()
        params = self.sinus_params()
        if self.sinus["mesh"] is not None:
            path = self.sinus["mesh"]
            if not os.path.isabs(path) and not os.path.exists(path):
                path = os.path.join(self.base_dir, path)
            sdf_dx = min(self.sinus["model_resolution_mm"] * MM, sim_dx)
            auto_needle, auto_outlet = None, None
            res = dict(sinus=None, mesh_path=path, sdf_dx=sdf_dx, mesh_padding=3.0 * sim_dx)
        else:
            mn, mx = params.bounds()
            dx = self.sinus["model_resolution_mm"] * MM
            size = [mx[i] - mn[i] for i in range(3)]
            dims = tuple(int(math.ceil(size[i] / dx)) + 1 for i in range(3))
            sx, sz = params.socket_xz
            yb = params.socket_bottom_y()
            r = params.socket_radius + 1.5 * sim_dx
            auto_outlet = ((sx - r, yb - 2.0 * sim_dx, sz - r), (sx + r, yb + 1.5 * sim_dx, sz + r))
            auto_needle = params.suggested_needle()
            res = dict(sinus=params, mesh_path=None, sdf_origin=tuple(mn), sdf_dx=dx, sdf_dims=dims)
        needle = self.resolve_needle(auto_needle)
        outlet = auto_outlet
        if self.outlet is not None:
            outlet = (tuple(x * MM for x in self.outlet["min_mm"]),
                      tuple(x * MM for x in self.outlet["max_mm"]))
        frames = max(self.sim["frames"], 1)
        frame_dt = self.sim["duration_s"] / frames
        return ResolvedScene(sim_dx=sim_dx, fluid=fluid, needle=needle, outlet=outlet,
                             solve=SolveParams(self.sim["pcg_iters"], self.sim["pcg_tol"]),
                             frames=frames, frame_dt=frame_dt, **res)


def load_stl(path: str):
    """Binary STL reader (mesh.rs:383-424): returns float64 triangles [T, 9] in file units."""
    import numpy as np
    with open(path, "rb") as f:
        buf = f.read()
    if len(buf) < 84:
        raise SceneError("STL file too small to be valid binary STL")
    n = int.from_bytes(buf[80:84], "little")
    if buf.startswith(b"solid") and len(buf) != 84 + 50 * n:
        raise SceneError("ASCII STL is not supported; re-export as binary STL")
    if len(buf) < 84 + 50 * n:
        raise SceneError(f"binary STL truncated: expected {84 + 50 * n} bytes, got {len(buf)}")
    rec = np.frombuffer(buf, dtype=np.uint8, count=50 * n, offset=84).reshape(n, 50)
    v = rec[:, 12:48].copy().view("<f4").reshape(n, 9)
    return v.astype(np.float64)


def load_obj(path: str):
    """Wavefront OBJ reader (mesh.rs:301-353): fan-triangulated float64 triangles [T, 9]."""
    import numpy as np
    verts, tris = [], []
    with open(path) as f:
        for line in f:
            tok = line.strip().split()
            if not tok:
                continue
            if tok[0] == "v":
                c = [float(t) for t in tok[1:4]]
                if len(c) < 3:
                    raise SceneError(f"malformed vertex line: {line!r}")
                verts.append(c)
            elif tok[0] == "f":
                face = [int(t.split("/")[0]) for t in tok[1:]]
                if len(face) < 3:
                    raise SceneError(f"face with fewer than 3 vertices: {line!r}")
                idx = [i - 1 if i > 0 else len(verts) + i for i in face]
                for k in range(1, len(idx) - 1):
                    tris.append(verts[idx[0]] + verts[idx[k]] + verts[idx[k + 1]])
    return np.array(tris, dtype=np.float64).reshape(-1, 9)


def load_mesh(path: str):
    """TriMesh::load (mesh.rs:272-283), dispatch on extension."""
    ext = os.path.splitext(path)[1].lower()
    if ext == ".stl":
        return load_stl(path)
    if ext == ".obj":
        return load_obj(path)
    raise SceneError(f"unsupported mesh extension: {ext!r} (use .obj or .stl)")
