"""Shared GPU-test fixtures: small scenes, identical-state setup for shadow stepping."""
from __future__ import annotations

import json
import os

import numpy as np

import oracle
from sdr_b200 import scene as sc
from tests.helpers import oracle_solver

# Folder for the parity statistics of the GPU tests (diagnostic output; not
# written unless SDR_TEST_RECORD_DIR is set).
OUT = os.environ.get("SDR_TEST_RECORD_DIR")

SMOKE_TOML = """
[sim]
resolution_mm = 2.0
duration_s = 0.5
frames = 10
[needle]
auto = true
diameter_mm = 0.8
flow_rate_ml_s = 5.0
[fluid]
particles_per_cell = 8
"""


def record(name: str, data: dict) -> None:
    """Append parity statistics to parity.json in SDR_TEST_RECORD_DIR, if set."""
    if not OUT:
        return
    os.makedirs(OUT, exist_ok=True)
    path = os.path.join(OUT, "parity.json")
    all_ = {}
    if os.path.exists(path):
        try:
            all_ = json.load(open(path))
        except Exception:
            all_ = {}
    all_[name] = data
    with open(path, "w") as f:
        json.dump(all_, f, indent=1, default=float)


def f32(a: np.ndarray) -> np.ndarray:
    """Round to f32 and widen back: the exact values the device stores."""
    return np.asarray(a, dtype=np.float64).astype(np.float32).astype(np.float64)


def make_pair(toml: str = SMOKE_TOML, warm_frames: int = 0, warm_dt: float | None = None):
    """A GPU solver and an oracle solver on the same SDF and parameters.

    The oracle is stepped ``warm_frames`` frames to reach a state with fluid,
    then both take that state rounded to f32 (identical inputs)."""
    from sdr_b200.solver import Sdf, Solver
    cfg = sc.SceneConfig.from_toml_str(toml)
    res = cfg.resolve()
    osdf = oracle.sdf_from_sinus(res.sinus, res.sdf_origin, res.sdf_dx, res.sdf_dims)
    orc = oracle_solver(res, osdf)
    for _ in range(warm_frames):
        orc.step(warm_dt if warm_dt is not None else res.frame_dt)
    gpu = Solver(Sdf(tuple(osdf.origin), osdf.dx, osdf.data.copy()), res.sim_dx, res.fluid, res.needle)
    gpu.solve = res.solve
    gpu.outlet = res.outlet
    pos, vel = orc.particles()
    pos, vel = f32(pos), f32(vel)
    orc.set_particles(pos, vel)
    gpu.set_particles(pos, vel)
    s = orc.scalars()
    gpu.set_scalars(s["time"], s["emit_accum"], s["steps"], s["drained"], s["rng"])
    return gpu, orc, res


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    scale = max(float(np.max(np.abs(b))) if b.size else 0.0, 1e-30)
    return float(np.max(np.abs(a - b))) / scale if a.size else 0.0
