"""Named workloads: the scenes the benchmark and scaling runs are quoted on.

plain_parametric  the `sdr init` parametric sinus at 0.8 mm, 4 ml/s for 0.5 s (52x55x41 cells)
real_cavity       seeded perturbed-ellipsoid cavity (2.2 ml, ~20k triangles, SH noise 15 %),
                  winding-number SDF at 0.5 mm; a 1 ml dose (4 ml/s for 0.25 s) then 0.35 s of
                  settling, 18 frames (the real-cavity shape stood in for by synthetic input)
large_parametric  the parametric sinus at 0.2 mm (207x217x161 cells), 6 ml/s for 0.3 s then
                  0.3 s settling, PCG capped at 400 iterations
batch_scene(seed) one scene of the batched / served family: a seeded perturbed ellipsoid of
                  U[1.5, 3] ml, grid cells log-uniform in [32^3, 96^3], needle tilt U[-30, 30] deg,
                  flow U[1, 8] ml/s, dose U[0.5, 2] ml, 0.6 s in 18 frames
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import scene as sc
from .cavity import perturbed_ellipsoid


@dataclass
class Workload:
    name: str
    res: sc.ResolvedScene
    tris: Optional[np.ndarray] = None   # mesh cavities
    cavity_volume: Optional[float] = None
    describe: Optional[dict] = None


def plain_parametric() -> Workload:
    cfg = sc.SceneConfig.from_toml_str(
        "[sim]\nresolution_mm = 0.8\nduration_s = 0.5\nframes = 15\npcg_tol = 1e-6\n"
        "[needle]\nflow_rate_ml_s = 4.0\n")
    return Workload("plain_parametric", cfg.resolve(),
                    describe={"cavity": "parametric sinus (sdr init defaults)", "dx_mm": 0.8,
                              "flow_ml_s": 4.0, "duration_s": 0.5})


def large_parametric() -> Workload:
    cfg = sc.SceneConfig.from_toml_str(
        "[sim]\nresolution_mm = 0.2\nduration_s = 0.6\nframes = 18\npcg_iters = 400\npcg_tol = 1e-6\n"
        "[needle]\nflow_rate_ml_s = 6.0\ninject_s = 0.3\n")
    return Workload("large_parametric", cfg.resolve(),
                    describe={"cavity": "parametric sinus", "dx_mm": 0.2, "flow_ml_s": 6.0,
                              "inject_s": 0.3, "duration_s": 0.6, "pcg_iters": 400})


def real_cavity(seed: int = 2, tilt_deg: float = 0.0, flow_ml_s: float = 4.0, dose_ml: float = 1.0,
                volume_ml: float = 2.2, dx_mm: float = 0.5, duration_s: float = 0.6, frames: int = 18) -> Workload:
    cav = perturbed_ellipsoid(seed, volume_ml=volume_ml, tilt_deg=tilt_deg)
    sim_dx = dx_mm * sc.MM
    fluid = sc.FluidParams(density=1000.0, gravity=(0.0, -9.81, 0.0), flip_ratio=0.7, particles_per_cell=8,
                           volume_stiffness=1.0, redistribute=True, redist_cap_factor=1.0)
    needle = sc.Needle(tip=cav.tip, axis=cav.axis, radius=0.5 * 0.8 * sc.MM, flow_rate=flow_ml_s * sc.ML_PER_S,
                       inject_until=dose_ml / flow_ml_s)
    res = sc.ResolvedScene(sim_dx=sim_dx, fluid=fluid, needle=needle, outlet=None,
                           solve=sc.SolveParams(200, 1e-6), frames=frames, frame_dt=duration_s / frames,
                           sinus=None, mesh_path=None, sdf_dx=sim_dx, mesh_padding=3.0 * sim_dx)
    return Workload("real_cavity", res, tris=cav.tris, cavity_volume=abs(cav.volume),
                    describe={"cavity": f"perturbed ellipsoid seed {seed}, {len(cav.tris)} triangles, "
                                        f"{volume_ml} ml, SH degree 1-4 noise 15%",
                              "dx_mm": dx_mm, "flow_ml_s": flow_ml_s, "dose_ml": dose_ml,
                              "duration_s": duration_s, "tilt_deg": tilt_deg})


def batch_scene(seed: int, frames: Optional[int] = None) -> Workload:
    """One scene of the batched family, every choice drawn from SplitMix64(seed).

    The cell size follows from the target cell count over the cavity's
    bounding box: dx = (bbox volume / N)^(1/3). ``frames`` shortens the run
    (the frame length stays 0.6 s / 18)."""
    from .cavity import SplitMix64
    rng = SplitMix64(0x5CE7E000 + seed)
    volume_ml = rng.uniform(1.5, 3.0)
    cells = math.exp(rng.uniform(math.log(32.0 ** 3), math.log(96.0 ** 3)))
    tilt = rng.uniform(-30.0, 30.0)
    flow = rng.uniform(1.0, 8.0)
    dose = rng.uniform(0.5, 2.0)
    cav = perturbed_ellipsoid(seed, volume_ml=volume_ml, tilt_deg=tilt)
    pts = cav.tris.reshape(-1, 3)
    ext = pts.max(axis=0) - pts.min(axis=0)
    dx = float((ext[0] * ext[1] * ext[2] / cells) ** (1.0 / 3.0))
    fluid = sc.FluidParams(density=1000.0, gravity=(0.0, -9.81, 0.0), flip_ratio=0.7, particles_per_cell=8,
                           volume_stiffness=1.0, redistribute=True, redist_cap_factor=1.0)
    needle = sc.Needle(tip=cav.tip, axis=cav.axis, radius=0.5 * 0.8 * sc.MM, flow_rate=flow * sc.ML_PER_S,
                       inject_until=dose / flow)
    total = 18
    res = sc.ResolvedScene(sim_dx=dx, fluid=fluid, needle=needle, outlet=None, solve=sc.SolveParams(200, 1e-6),
                           frames=total if frames is None else int(frames), frame_dt=0.6 / total, sinus=None,
                           mesh_path=None, sdf_dx=dx, mesh_padding=3.0 * dx)
    return Workload(f"batch_scene_{seed}", res, tris=cav.tris, cavity_volume=abs(cav.volume),
                    describe={"seed": seed, "volume_ml": volume_ml, "target_cells": cells, "dx_mm": dx * 1e3,
                              "tilt_deg": tilt, "flow_ml_s": flow, "dose_ml": dose})


def scene_spec(w: Workload):
    """The batched-run description of a workload (its SDF voxelised on the device)."""
    from .serving import SceneSpec
    from .solver import build_sdf, cavity_volume
    sdf = build_sdf(w.res, w.tris)
    vol = w.cavity_volume if w.cavity_volume is not None else cavity_volume(w.res, sdf, w.tris)
    return SceneSpec(sdf=sdf, sim_dx=w.res.sim_dx, fluid=w.res.fluid, needle=w.res.needle, solve=w.res.solve,
                     cavity_volume=vol, frame_dt=w.res.frame_dt, frames=w.res.frames, outlet=w.res.outlet)


WORKLOADS = {"plain_parametric": plain_parametric, "real_cavity": real_cavity, "large_parametric": large_parametric}


def hash_jitter(keys: np.ndarray) -> np.ndarray:
    """hash_jitter (solver.rs:916-930) for an array of u64 keys: a splitmix64
    finaliser of 3k, 3k+1, 3k+2, the top 53 bits mapped to [-0.3, 0.3); (n, 3) f64."""
    k3 = np.asarray(keys, dtype=np.uint64) * np.uint64(3)
    out = np.empty((k3.shape[0], 3))
    for c in range(3):
        z = k3 + np.uint64(c) + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z ^= z >> np.uint64(31)
        out[:, c] = ((z >> np.uint64(11)).astype(np.float64) / float(1 << 53) - 0.5) * 0.6
    return out


def preseed_pool(solver, target: int, ppc: int = 8):
    """Pre-seeded pool: the lowest in-cavity cells along gravity (ties in cell
    order), ``ppc`` particles each at the cell centre plus hash_jitter(index) * dx,
    at rest, until ``target`` particles or the cavity is full. Returns (pos, vel)
    in f64 for ``Solver.set_particles``."""
    st = solver.stats()
    return preseed_pool_on((int(st.nx), int(st.ny), int(st.nz)), (st.origin.x, st.origin.y, st.origin.z),
                           float(st.dx), solver.fluid.gravity, solver.cavity_mask(), target, ppc)


def preseed_pool_on(dims, origin, dx: float, gravity, cavity_mask: np.ndarray, target: int, ppc: int = 8):
    """preseed_pool from the grid, gravity and static cavity mask alone (the
    same particles for any solver holding that grid)."""
    nx, ny, nz = (int(v) for v in dims)
    dx = float(dx)
    org = np.array(origin, dtype=np.float64)
    g = np.array(gravity, dtype=np.float64)
    cav = np.flatnonzero(np.asarray(cavity_mask).reshape(-1))
    i = cav % nx
    j = (cav // nx) % ny
    k = cav // (nx * ny)
    centre = org + (np.stack([i, j, k], axis=1) + 0.5) * dx
    gl = np.linalg.norm(g)
    depth = centre @ (g / gl) if gl > 0 else np.zeros(len(cav))
    order = np.argsort(-depth, kind="stable")  # deepest along gravity first
    ncell = min(len(cav), -(-int(target) // ppc))
    cells = order[:ncell]
    n = min(int(target), ncell * ppc)
    idx = np.arange(n, dtype=np.uint64)
    pos = centre[cells].repeat(ppc, axis=0)[:n] + hash_jitter(idx) * dx
    return pos, np.zeros_like(pos)


def build_gpu(w: Workload, max_particles: int = 0):
    """Device SDF + solver for a workload; returns (solver, sdf, cavity_volume)."""
    from .solver import Solver, build_sdf, cavity_volume
    sdf = build_sdf(w.res, w.tris)
    vol = w.cavity_volume if w.cavity_volume is not None else cavity_volume(w.res, sdf, w.tris)
    s = Solver(sdf, w.res.sim_dx, w.res.fluid, w.res.needle, max_particles=max_particles)
    s.solve = w.res.solve
    s.outlet = w.res.outlet
    return s, sdf, vol
