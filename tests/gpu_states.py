"""Identical GPU and oracle states on the benchmark workloads (shadow stepping).

Each state is reached on the device (fast), then copied into the oracle: the
particles as the device stores them (f32, widened to f64) and the solver's
scalars (time, emission accumulator, rng, drained, steps). From there one
phase, or one whole substep, runs on both and the outputs are compared.

  smoke_2mm             the CI smoke scene (parametric sinus, 2 mm), 3 oracle frames
  parametric_0p8mm      the `sdr init` parametric sinus at 0.8 mm, 4 ml/s (52x55x41
                        cells), after 3 frames of the jet (0.1 s)
  cavity_0p5mm_jet      perturbed-ellipsoid cavity (2.2 ml, 20,480 triangles) at 0.5 mm,
                        1 ml at 4 ml/s, after 4 frames (0.13 s, jet firing)
  cavity_0p5mm_settled  the same cavity after 12 frames (0.4 s, dose in, settling)
  pool_0p2mm            the parametric sinus at 0.2 mm (207x217x161 cells) holding a
                        pre-seeded pool of 9.5 M particles, after 2 substeps at the
                        jet CFL step
"""
from __future__ import annotations

import numpy as np

import oracle
from sdr_b200 import workloads
from tests.gpu_common import SMOKE_TOML, f32, make_pair
from tests.helpers import oracle_solver

STATES = ("smoke_2mm", "parametric_0p8mm", "cavity_0p5mm_jet", "cavity_0p5mm_settled", "pool_0p2mm")


def gpu_to_oracle(gpu, orc) -> None:
    """Copy the device's particle set and scalars into the oracle."""
    pos, vel = gpu.particles()
    orc.set_particles(pos, vel)
    st = gpu.stats()
    orc.set_scalars(st.time, st.emit_accum, st.steps, st.drained, st.rng_state)


def sync_faces(gpu, orc, which=(0, 1, 2, 3, 4, 5)) -> None:
    for w in which:
        orc.set_face(w, gpu.face(w))


def _pair_on(w: workloads.Workload, sdf_data_from_oracle: bool, max_particles: int = 0):
    from sdr_b200.solver import Sdf, Solver, build_sdf
    res = w.res
    if sdf_data_from_oracle:  # parametric: the oracle's implicit field, handed to both
        osdf = oracle.sdf_from_sinus(res.sinus, res.sdf_origin, res.sdf_dx, res.sdf_dims)
        sdf = Sdf(tuple(osdf.origin), osdf.dx, osdf.data.copy())
    else:  # mesh: the device's winding-number SDF (bit-exact with the oracle's), handed to both
        sdf = build_sdf(res, w.tris)
        osdf = oracle.SdfGrid(tuple(sdf.origin), sdf.dx, sdf.data)
    gpu = Solver(sdf, res.sim_dx, res.fluid, res.needle, max_particles=max_particles)
    gpu.solve = res.solve
    gpu.outlet = res.outlet
    orc = oracle_solver(res, osdf)
    return gpu, orc, res


def make_state(name: str):
    """(gpu, orc, res) holding the same state; see the module docstring."""
    if name == "smoke_2mm":
        return make_pair(SMOKE_TOML, warm_frames=3)
    if name == "parametric_0p8mm":
        gpu, orc, res = _pair_on(workloads.plain_parametric(), True)
        for _ in range(3):
            gpu.step(res.frame_dt)
    elif name in ("cavity_0p5mm_jet", "cavity_0p5mm_settled"):
        gpu, orc, res = _pair_on(workloads.real_cavity(seed=2), False)
        for _ in range(4 if name.endswith("jet") else 12):
            gpu.step(res.frame_dt)
    elif name == "pool_0p2mm":
        gpu, orc, res = _pair_on(workloads.large_parametric(), True, max_particles=12_000_000)
        pos, vel = workloads.preseed_pool(gpu, 30_000_000)
        gpu.set_particles(f32(pos), vel)
        jet = gpu.needle.flow_rate / (np.pi * gpu.needle.radius ** 2)
        for _ in range(2):
            gpu.substep(gpu.dx / jet)
    else:
        raise KeyError(name)
    gpu_to_oracle(gpu, orc)
    return gpu, orc, res
