#!/usr/bin/env python
"""Benchmark: particle-substeps/s of the FLIP/PIC substep on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl sdr|reference]

Headline (``value``): the largest single-GPU workload, ``pool_0p2mm`` - the
`sdr init` parametric sinus at 0.2 mm (207 x 217 x 161 = 7.23 M cells, 6 ml/s
jet, PCG capped at 400 iterations) holding a pre-seeded pool of 9.5 M
particles at rest (the deepest cavity cells filled at 8 particles per cell
with hash_jitter offsets). A step is one Solver::substep at the jet's CFL step
(dx / jet speed). W warm-up substeps run from the pre-seeded state, then the
state is put back (particles and scalars) and K substeps are timed from it, so
the timed window is the same for every run and for the reference arm. The
state (1.5 GB on the device) is far larger than the 126 MB L2, so no flush is
needed between steps.

``value`` is device time: CUDA events on the solver stream around every
substep, summed, max over ranks. ``e2e`` times the same substeps on the host
around the public call (sdr_solver_substep: the emitted particles' host ->
device upload and the device -> host status read of every substep inside).

``--impl reference`` times the CPU restatement of the reference solver
(oracle/; the reference is Rust and cannot be built here) on all host threads,
from the identical pre-seeded state at the same dt: a bounded sample of the
first ``--ref-substeps`` substeps of the window (one oracle substep takes
~14 s on 16 threads).

Extra records on one GPU:
``parametric_0p8mm`` the parametric sinus at 0.8 mm, 4 ml/s, the whole 0.5 s
                   (15 frames) timed frame by frame after a warm-up run, with
                   the per-frame read-back of positions; the oracle continues
                   from the mid-run state for a bounded sample.
``cavity_0p5mm``   the perturbed-ellipsoid cavity (2.2 ml, 20,480 triangles,
                   winding-number SDF at 0.5 mm), 1 ml at 4 ml/s, the whole
                   0.6 s (18 frames), timed the same way.
``batched``/``served`` a bounded sample of the batched scene family (seeded
                   perturbed-ellipsoid cavities, grids log-uniform in
                   32^3..96^3 cells, needle tilt, flow and dose drawn per
                   scene): one after another on default solvers (the plain
                   path), all at once (sdr_batch_run), and as Poisson
                   arrivals into the request server with p50/p99
                   time-to-summary.
``render``         preview images (600 px) of the cavity run's final state
                   beside the oracle drawing the same state.

``--batched-full`` runs only the batched family at full duration instead:
128 scenes for 0.6 s each, all at once (packed, then stream per scene) against
a seeded plain sample of 8 of them, then 32 Poisson requests (90 % family,
10 % the real-cavity scene) into both request servers against a plain sample
of the requests; each phase prints a line as it ends, then the summary line
(scenes/s).

Multi-GPU runs are independent replicas (one pool per rank): no collective on
the data path; a barrier and a max-reduce of the timings use torch.distributed.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
# Concurrent scenes use one CUDA stream each: give the device more hardware
# queues than the default 8 (read when the CUDA context is created).
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

# Algorithmic bytes of the pressure solve (the dominant kernel), f64 vectors in
# wavefront order: per fluid cell and PCG iteration (matvec 41, dot 20, p/r
# update 48, forward sweep 44, backward sweep 36, second dot 20, direction 24)
# and per fluid cell once per solve (factorisation, first preconditioner
# application, setup).
PCG_BYTES_PER_CELL_ITER = 233
PCG_BYTES_PER_CELL_SOLVE = 190
POOL_TARGET = 30_000_000   # particles asked for; the cavity holds 9.5 M at 8 per cell
POOL_CAPACITY = 12_000_000


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    return int(os.environ.get("RANK", "0")), ws, int(os.environ.get("LOCAL_RANK", "0"))


def substep_bytes(particle_substeps: int, substeps: int, cells: int, sdf_nodes: int, cell_iters: int) -> float:
    """Algorithmic bytes of `substeps` substeps by the per-substep contract
    B = 112 P + 92 C + 4 S + 83 N_f iters (f32 particle and face state, u8
    labels, f32 solve vectors, f64 factor): P particles, C grid cells, S SDF
    nodes, N_f fluid cells; summed over substeps."""
    return 112.0 * particle_substeps + (92.0 * cells + 4.0 * sdf_nodes) * substeps + 83.0 * cell_iters


def reduce_over_ranks(dev_ms: float, wall: float, ps: int, device: str):
    """Whole-job figures of a multi-rank run: the slowest rank's device and
    wall time (max) and the particle-substeps of all ranks (sum). Every rank
    takes the same two collectives in the same order."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([dev_ms, wall], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([float(ps)], dtype=torch.float64, device=device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t[0]), float(t[1]), int(c[0])


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measured_traffic(kernel: str, workload: str):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of
    this kernel on this workload from the committed ncu summaries, or None."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    return json.load(open(p)).get(f"{kernel}@{workload}")


class Clocks:
    """nvidia-smi sampler for the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows if len(r) >= 9 for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------- the pool workload
def pool_config(w, grid, particles: int, dt: float) -> dict:
    """The headline's config, identical in both arms."""
    return {"workload": "pool_0p2mm", "cavity": "parametric sinus (sdr init defaults)", "dx_mm": 0.2,
            "grid": [int(v) for v in grid], "particles": int(particles),
            "state": "pre-seeded pool at rest, 8 particles per cell (hash_jitter offsets), deepest cavity cells first",
            "flow_ml_s": 6.0, "dt_s": dt, "dt_rule": "jet CFL step dx / jet speed",
            "pcg_iters_cap": int(w.res.solve.max_iters), "pcg_tol": float(w.res.solve.tol),
            "window": "substeps 1..K from the pre-seeded state",
            "l2": "state 1.5 GB, larger than the 126 MB L2 (no flush)"}


def jet_dt(needle, dx: float) -> float:
    import math
    return dx / (needle.flow_rate / (math.pi * needle.radius ** 2))


def oracle_for(w, sdf):
    import oracle
    from tests.helpers import oracle_solver
    osdf = oracle.SdfGrid(tuple(sdf.origin), sdf.dx, sdf.data)
    return oracle_solver(w.res, osdf)


def run_reference(args):
    """The oracle on the host cores: the pre-seeded pool, the same dt, the first
    --ref-substeps substeps of the GPU arm's window."""
    import numpy as np

    import oracle
    from sdr_b200 import workloads
    from tests.helpers import oracle_solver
    w = workloads.large_parametric()
    res = w.res
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    osdf = oracle.sdf_from_sinus(res.sinus, res.sdf_origin, res.sdf_dx, res.sdf_dims)
    orc = oracle_solver(res, osdf)
    (nx, ny, nz), origin, dx = orc.grid
    pos, vel = workloads.preseed_pool_on((nx, ny, nz), origin, dx, res.fluid.gravity, orc.cavity_mask(),
                                         POOL_TARGET)
    pos = pos.astype(np.float32).astype(np.float64)
    orc.set_particles(pos, vel)
    dt = jet_dt(res.needle, dx)
    n_sub = max(1, min(args.steps, args.ref_substeps))
    ps, t = 0, 0.0
    for _ in range(n_sub):
        ps += len(orc)
        t0 = time.perf_counter()
        orc.substep(dt)
        t += time.perf_counter() - t0
    v = ps / t
    sample = (f"the first {n_sub} substeps of the timed window from the identical pre-seeded state "
              f"({ps} particle-substeps, {t:.1f} s); C++ restatement of the reference solver (the Rust "
              "reference cannot be built here), f64, rayon-parallel parts on all host threads")
    line = {"metric": "particle-substeps/s", "value": v, "unit": "particle-substeps/s", "impl": "reference",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / n_sub,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": pool_config(w, (nx, ny, nz), len(pos), dt),
            "cpu_baseline": {"value": v, "unit": "particle-substeps/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": "particle-substeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def pool_line(args, rank, world, local):
    """The headline measurement (see the module docstring)."""
    import numpy as np
    import torch

    from sdr_b200 import _lib, workloads
    w = workloads.large_parametric()
    t0 = time.perf_counter()
    solver, sdf, vol = workloads.build_gpu(w, max_particles=POOL_CAPACITY)
    pos, vel = workloads.preseed_pool(solver, POOL_TARGET)
    pos = pos.astype(np.float32).astype(np.float64)  # the stored (f32) state, shared with the oracle
    setup_s = time.perf_counter() - t0
    dt = jet_dt(solver.needle, solver.dx)
    st_init = solver.stats()

    def reset():
        solver.set_particles(pos, vel)
        solver.set_scalars(st_init.time, st_init.emit_accum, st_init.steps, st_init.drained, st_init.rng_state)

    solver.set_profiling(True)
    reset()
    for _ in range(args.warmup):
        solver.substep(dt)
    reset()
    solver.reset_profile()
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    launches0 = _lib.load().sdr_kernel_launch_count()
    clk = Clocks(local)
    st0 = solver.stats()
    wall = 0.0
    for _ in range(args.steps):
        t1 = time.perf_counter()
        solver.substep(dt)  # public call: emission upload and status read inside
        wall += time.perf_counter() - t1
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = clk.stop()
    st1 = solver.stats()
    launches = _lib.load().sdr_kernel_launch_count() - launches0
    prof = solver.profile()
    dev_ms = st1.device_ms - st0.device_ms
    local_dev_ms = dev_ms
    ps = st1.particle_substeps - st0.particle_substeps
    if world > 1:
        dev_ms, wall, ps = reduce_over_ranks(dev_ms, wall, ps, "cuda")
    value = ps / (dev_ms / 1e3)
    e2e = ps / wall
    hbm, peak_kind = peaks()
    n_pcg = max(prof["pcg_launches"], 1)
    if prof.get("pcg_tile_launches", 0) == prof["pcg_launches"]:
        kernel = "k_pcg_tiles"
    elif prof["pcg_cluster_launches"] == prof["pcg_launches"]:
        kernel = "k_pcg_cluster"
    else:
        kernel = "k_pcg"
    pcg_launch_ms = prof["pcg_ms"] / n_pcg
    pcg_bytes = (PCG_BYTES_PER_CELL_ITER * prof["pcg_cell_iters"] + PCG_BYTES_PER_CELL_SOLVE * prof["fluid_cells"]) / n_pcg
    achieved = pcg_bytes / (pcg_launch_ms / 1e3) / 1e9 if pcg_launch_ms > 0 else 0.0
    traffic = measured_traffic(kernel, "pool_0p2mm")
    sub_bytes = substep_bytes(prof["particles"], prof["substeps"], int(st1.nx * st1.ny * st1.nz),
                              int(sdf.data.size), prof["pcg_cell_iters"])
    sub_gbs = sub_bytes / (local_dev_ms / 1e3) / 1e9 if local_dev_ms > 0 else 0.0  # this rank's substeps
    line = {"metric": "particle-substeps/s", "value": value, "unit": "particle-substeps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic", "config": pool_config(w, (st1.nx, st1.ny, st1.nz), len(pos), dt),
            "e2e": {"value": e2e, "unit": "particle-substeps/s",
                    "h2d_bytes_per_step": int(prof["h2d_bytes"] / args.steps),
                    "d2h_bytes_per_step": int(prof["d2h_bytes"] / args.steps)},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "roofline": {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "peak_kind": peak_kind,
                         "traffic": traffic["bytes_per_launch"] if traffic else None,
                         "traffic_source": traffic["source"] if traffic else None,
                         "bytes_per_launch": pcg_bytes, "ms_per_launch": pcg_launch_ms,
                         "bytes": f"{PCG_BYTES_PER_CELL_ITER} B per fluid cell per iteration + "
                                  f"{PCG_BYTES_PER_CELL_SOLVE} B per fluid cell per solve"},
            "substep_roofline": {"bound": "hbm", "achieved": sub_gbs, "peak": hbm, "unit": "GB/s",
                                 "frac": sub_gbs / hbm, "peak_kind": peak_kind,
                                 "bytes_per_substep": sub_bytes / max(prof["substeps"], 1),
                                 "bytes": "112 P + 92 C + 4 S + 83 N_f iters per substep"},
            "phase_ms_per_substep": {k: round(v / max(prof["substeps"], 1), 3) for k, v in prof.items()
                                     if k.endswith("_ms")},
            "pcg": {"launches": prof["pcg_launches"], "kernel": kernel,
                    "mean_iters": prof["pcg_cell_iters"] / max(prof["fluid_cells"], 1),
                    "mean_fluid_cells": prof["fluid_cells"] / n_pcg},
            "redistribution": {"candidates": prof["redist_candidates"], "sweeps": prof["redist_sweeps"],
                               "long_sweeps": prof["redist_long_sweeps"], "rounds": prof["redist_rounds"]},
            "setup_s": setup_s}
    if rank == 0 and world == 1 and not args.no_cpu:
        import oracle
        threads = os.cpu_count() or 1
        oracle.set_threads(threads)
        orc = oracle_for(w, sdf)
        orc.set_particles(pos, vel)
        t1 = time.perf_counter()
        orc.substep(dt)
        ct = time.perf_counter() - t1
        line["cpu_baseline"] = {"value": len(pos) / ct, "unit": "particle-substeps/s", "cores": threads,
                                "kind": "port", "sample": f"substep 1 of the timed window from the identical "
                                                          f"pre-seeded state ({ct:.1f} s); C++ restatement of the "
                                                          "reference solver, f64, on all host threads"}
        del orc
    solver.close()
    return line


# ---------------------------------------------------------------- frame-based runs
def frame_record(w, key: str, cpu: bool, cpu_budget: float):
    """A whole run of a scene (every frame) timed frame by frame after a
    warm-up run of two frames on another solver; between frames a 256 MiB
    buffer is written to flush L2 (these states are smaller than L2)."""
    import torch

    from sdr_b200 import workloads
    warm, _, _ = workloads.build_gpu(w)
    for _ in range(2):
        warm.step(w.res.frame_dt)
    warm.close()
    solver, sdf, vol = workloads.build_gpu(w)
    solver.set_profiling(True)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    dev_ms = wall = 0.0
    ps = 0
    mid = None
    for f in range(w.res.frames):
        flush.zero_()
        torch.cuda.synchronize()
        st0 = solver.stats()
        t0 = time.perf_counter()
        solver.step(w.res.frame_dt)
        pos, _ = solver.particles_f32()  # the per-frame read-back of cmd_simulate's output
        wall += time.perf_counter() - t0
        st1 = solver.stats()
        dev_ms += st1.device_ms - st0.device_ms
        ps += st1.particle_substeps - st0.particle_substeps
        if f == w.res.frames // 2 and cpu:
            p, v = solver.particles()
            mid = (p, v, st1)
    prof = solver.profile()
    st = solver.stats()
    out = {"workload": key, **(w.describe or {}), "grid": [st.nx, st.ny, st.nz], "frames": w.res.frames,
           "substeps": int(prof["substeps"]), "particles_end": int(st.particles),
           "particle_substeps_per_s": ps / (dev_ms / 1e3), "e2e_particle_substeps_per_s": ps / wall,
           "device_s": dev_ms / 1e3, "wall_s": wall,
           "phase_ms": {k: round(v, 3) for k, v in prof.items() if k.endswith("_ms")},
           "pcg": {"mean_iters": prof["pcg_cell_iters"] / max(prof["fluid_cells"], 1),
                   "mean_fluid_cells": prof["fluid_cells"] / max(prof["pcg_launches"], 1)},
           "redistribution": {"candidates": prof["redist_candidates"], "sweeps": prof["redist_sweeps"]},
           "mass": {"emitted": st.emitted, "resident": st.particles, "drained": st.drained, "culled": st.culled}}
    if cpu and mid is not None:
        import oracle
        threads = os.cpu_count() or 1
        oracle.set_threads(threads)
        orc = oracle_for(w, sdf)
        p, v, s = mid
        orc.set_particles(p, v)
        orc.set_scalars(s.time, s.emit_accum, s.steps, s.drained, s.rng_state)
        t0 = time.perf_counter()
        cps = csub = 0
        while time.perf_counter() - t0 < cpu_budget:
            dt = orc.cfl_dt()
            cps += len(orc)
            orc.substep(dt)
            csub += 1
        ct = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": cps / ct, "unit": "particle-substeps/s", "cores": threads, "kind": "port",
                               "sample": f"{csub} substeps from the mid-run state (frame {w.res.frames // 2}), "
                                         f"{ct:.1f} s"}
        out["speedup_vs_cpu"] = out["particle_substeps_per_s"] / out["cpu_baseline"]["value"]
        out["e2e_speedup_vs_cpu"] = out["e2e_particle_substeps_per_s"] / out["cpu_baseline"]["value"]
    return {key: out}, solver, sdf


def _serve(specs, rate: float, seed: int, packed: bool) -> tuple:
    """Poisson arrivals at `rate` into the request server; (results, seconds, stats)."""
    import random

    from sdr_b200.serving import Server
    rng = random.Random(seed)
    with Server(budget_bytes=150 << 30, max_active=len(specs), packed=packed) as srv:
        t0 = time.perf_counter()
        tickets, t_next = [], 0.0
        for sp in specs:
            t_next += rng.expovariate(rate)
            delay = t0 + t_next - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            tickets.append(srv.submit(sp))
        res = srv.wait(tickets, timeout=3600)
        t_srv = time.perf_counter() - t0
        sst = srv.stats()
    return res, t_srv, sst


def batch_bench(n_scenes: int, cfl_steps: int, seed0: int = 100) -> dict:
    """The same scenes one after another on default solvers (the plain path),
    concurrently on one stream and solver each (sdr_batch_run), packed into one
    launch per substep operation (sdr_batch_run_packed), and served: Poisson
    arrivals into the request server, stream-per-scene and packed."""
    import math

    from sdr_b200 import _lib, workloads
    from sdr_b200.serving import run_batch
    t0 = time.perf_counter()
    specs = []
    for i in range(n_scenes):
        sp = workloads.scene_spec(workloads.batch_scene(seed0 + i, frames=1))
        jet = sp.needle.flow_rate / (math.pi * sp.needle.radius ** 2)
        sp.frame_dt = cfl_steps * sp.sim_dx / jet
        specs.append(sp)
    build_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    plain = run_batch(specs, concurrency=1)
    t_plain = time.perf_counter() - t0
    t0 = time.perf_counter()
    mix = run_batch(specs, concurrency=0)
    t_mix = time.perf_counter() - t0
    cnt = {}
    t0 = time.perf_counter()
    packed = run_batch(specs, packed=True, counters=cnt)
    t_packed = time.perf_counter() - t0
    ok = all(r.status == _lib.SDR_OK for r in plain + mix + packed)
    same = ok and all(a.summary == b.summary == c.summary for a, b, c in zip(plain, mix, packed))
    ps = sum(r.stats["particle_substeps"] for r in packed) if ok else 0
    subs = sum(r.stats["substeps_total"] for r in packed) if ok else 0
    best = min(t_mix, t_packed)
    rate = 0.8 * n_scenes / best  # arrivals at 80 % of the better batched throughput

    def served(packed_mode: bool) -> dict:
        res, t_srv, sst = _serve(specs, rate, seed0, packed_mode)
        lat = sorted(r.seconds for r in res)

        def pct(q):
            return lat[min(len(lat) - 1, int(round(q * (len(lat) - 1))))]
        return {"mode": "packed engine" if packed_mode else "one stream and host thread per scene",
                "arrivals": "poisson", "rate_per_s": rate, "scenes_per_s": n_scenes / t_srv,
                "p50_time_to_summary_s": pct(0.5), "p99_time_to_summary_s": pct(0.99),
                "peak_active": sst["peak_active"], "peak_bytes": sst["peak_bytes"], "budget_bytes": 150 << 30,
                "results_identical": ok and all(r.summary == b.summary for r, b in zip(res, plain))}
    sample = (f"{n_scenes} scenes of the batched family (seeds {seed0}..{seed0 + n_scenes - 1}), each one frame "
              f"of {cfl_steps} jet-CFL steps from t = 0; SDFs built on the device in {build_s:.1f} s")
    return {
        "batched": {"scenes": n_scenes, "cfl_steps_per_scene": cfl_steps, "sample": sample,
                    "plain_scenes_per_s": n_scenes / t_plain, "plain_s": t_plain,
                    "plain_solver": "default (sdr_solver_create flags 0), one scene after another",
                    "streams_scenes_per_s": n_scenes / t_mix, "streams_s": t_mix,
                    "packed_scenes_per_s": n_scenes / t_packed, "packed_s": t_packed,
                    "packed_counters": cnt,
                    "speedup_streams": t_plain / t_mix, "speedup_packed": t_plain / t_packed,
                    "particle_substeps_per_s_packed": ps / t_packed, "substeps": subs,
                    "results_identical": same},
        "served": served(False),
        "served_packed": served(True),
    }


def batched_full(n_scenes: int = 128, n_plain: int = 8, n_requests: int = 32, seed0: int = 100) -> dict:
    """The batched family at full duration (0.6 s, 18 frames per scene).

    Packed (one launch per substep operation for all scenes) and then one
    stream and solver per scene, all n_scenes at once. Plain: a seeded sample
    of n_plain of the same scenes one after another on default solvers (the
    whole family on the plain path would take about an hour); its time for all
    n_scenes is estimated as the sample's time x n_scenes / n_plain, and the
    sampled scenes' summaries must equal their batched ones. Served:
    n_requests Poisson arrivals, 90 % drawn from the family (new seeds) and
    10 % the real-cavity scene (0.5 mm, 1 ml), into both request servers at 80 %
    of the packed rate, against a plain sample of the same requests. Each phase
    prints a line ("phase": ...) as it ends."""
    import random

    from sdr_b200 import _lib, workloads
    from sdr_b200.serving import run_batch

    def say(**kw):
        print(json.dumps(kw), flush=True)
    t0 = time.perf_counter()
    specs = [workloads.scene_spec(workloads.batch_scene(seed0 + i)) for i in range(n_scenes)]
    build_s = time.perf_counter() - t0
    cnt = {}
    t0 = time.perf_counter()
    packed = run_batch(specs, packed=True, counters=cnt)
    t_packed = time.perf_counter() - t0
    ok = all(r.status == _lib.SDR_OK for r in packed)
    subs = sum(r.stats["substeps_total"] for r in packed) if ok else 0
    say(phase="packed", scenes=n_scenes, seconds=t_packed, scenes_per_s=n_scenes / t_packed, substeps=subs,
        counters=cnt, ok=ok)
    rng = random.Random(seed0)
    idx = sorted(rng.sample(range(n_scenes), n_plain))
    t0 = time.perf_counter()
    plain = run_batch([specs[i] for i in idx], concurrency=1)
    t_plain_sample = time.perf_counter() - t0
    t_plain_est = t_plain_sample * n_scenes / n_plain
    same_plain = all(r.status == _lib.SDR_OK for r in plain) and \
        all(p.summary == packed[i].summary for p, i in zip(plain, idx))
    say(phase="plain_sample", sample=idx, seconds=t_plain_sample, estimated_all_s=t_plain_est,
        results_identical=same_plain)
    t0 = time.perf_counter()
    mix = run_batch(specs, concurrency=0)
    t_mix = time.perf_counter() - t0
    same_mix = all(r.status == _lib.SDR_OK for r in mix) and \
        all(mix[i].summary == packed[i].summary for i in range(n_scenes))
    say(phase="streams", seconds=t_mix, scenes_per_s=n_scenes / t_mix, results_identical=same_mix)
    out = {"scenes": n_scenes, "frames_per_scene": 18, "duration_s": 0.6, "substeps": subs, "sdf_build_s": build_s,
           "packed_scenes_per_s": n_scenes / t_packed, "packed_s": t_packed, "packed_counters": cnt,
           "streams_scenes_per_s": n_scenes / t_mix, "streams_s": t_mix,
           "plain_sample": idx, "plain_sample_s": t_plain_sample, "plain_scenes_per_s": n_plain / t_plain_sample,
           "plain_estimated_s": t_plain_est,
           "speedup_packed": t_plain_est / t_packed, "speedup_streams": t_plain_est / t_mix,
           "results_identical": ok and same_plain and same_mix}
    rq = random.Random(seed0 + 1)
    reqs = []
    for q in range(n_requests):
        if rq.random() < 0.1:
            reqs.append(workloads.scene_spec(workloads.real_cavity(seed=2 + q)))
        else:
            reqs.append(workloads.scene_spec(workloads.batch_scene(seed0 + 1000 + q)))
    rate = 0.8 * n_scenes / t_packed
    pidx = sorted(rq.sample(range(n_requests), max(1, n_requests // 8)))
    t0 = time.perf_counter()
    pref = run_batch([reqs[i] for i in pidx], concurrency=1)
    t_pref = time.perf_counter() - t0
    srv = {"requests": n_requests, "mix": "90 % batched family, 10 % real cavity 0.5 mm", "rate_per_s": rate,
           "plain_sample": pidx, "plain_sample_s": t_pref, "plain_scenes_per_s": len(pidx) / t_pref}
    say(phase="served_plain_sample", **srv)
    for packed_mode in (True, False):
        res, t_srv, sst = _serve(reqs, rate, seed0, packed_mode)
        lat = sorted(r.seconds for r in res)

        def pct(q):
            return lat[min(len(lat) - 1, int(round(q * (len(lat) - 1))))]
        key = "packed" if packed_mode else "streams"
        srv[key] = {"scenes_per_s": n_requests / t_srv, "p50_time_to_summary_s": pct(0.5),
                    "p99_time_to_summary_s": pct(0.99), "peak_active": sst["peak_active"],
                    "peak_bytes": sst["peak_bytes"],
                    "results_identical": all(r.status == _lib.REQ_DONE for r in res) and
                    all(res[i].summary == p.summary for p, i in zip(pref, pidx))}
        say(phase="served_" + key, **srv[key])
    return {"batched_full": out, "served_full": srv}


def render_bench(solver, w, sdf, cpu: bool, px: int = 600, reps: int = 5) -> dict:
    """Preview images (render_slice) of the solver's current state: the slice
    through the needle tip (speed dots) and the gravity projection (amber
    pool), public call to host image; the oracle draws the same state."""
    from sdr_b200.render import SlicePlane, render_slice
    planes = {"slice": SlicePlane.xy(w.res.needle.tip[2], w.res.sim_dx),
              "gravity": SlicePlane.projected_along_gravity(w.res.fluid.gravity)}
    out = {"px": px, "particles": len(solver)}
    imgs = {}
    for name, plane in planes.items():
        imgs[name] = render_slice(solver, plane, px)  # warm-up
        t0 = time.perf_counter()
        for _ in range(reps):
            render_slice(solver, plane, px)
        out[f"{name}_ms"] = 1e3 * (time.perf_counter() - t0) / reps
    if cpu:
        orc = oracle_for(w, sdf)
        pos, vel = solver.particles()
        orc.set_particles(pos, vel)
        same = True
        for name, plane in planes.items():
            t0 = time.perf_counter()
            ref = orc.render_slice(plane.as_dict(), px)
            out[f"cpu_{name}_ms"] = 1e3 * (time.perf_counter() - t0)
            same = same and bool((ref == imgs[name]).all())
        out["identical_to_oracle"] = same
    return {"render": out}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="sdr", choices=["sdr", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=12.0, help="seconds of oracle time per extra record")
    ap.add_argument("--ref-substeps", type=int, default=4, help="substeps the reference arm times")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="headline only")
    ap.add_argument("--batch-scenes", type=int, default=48)
    ap.add_argument("--batch-cfl", type=int, default=150)
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--batched-full", action="store_true",
                    help="only the batched family at full duration and the serving mix (tens of minutes)")
    ap.add_argument("--full-scenes", type=int, default=128, help="scenes of --batched-full")
    ap.add_argument("--full-requests", type=int, default=32, help="served requests of --batched-full")
    args = ap.parse_args()
    rank, world, local = dist_env()

    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return

    import torch
    torch.cuda.set_device(local)
    if args.batched_full:
        if rank == 0:
            rec = batched_full(args.full_scenes, max(1, min(8, args.full_scenes // 16)), args.full_requests)
            print(json.dumps({"metric": "scenes/s", "value": rec["batched_full"]["packed_scenes_per_s"],
                              "unit": "scenes/s", "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
                              "config": {"workload": f"batched family x{args.full_scenes} at 0.6 s; serving mix"},
                              **rec}))
        return
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    line = pool_line(args, rank, world, local)
    if rank == 0 and world == 1 and not args.no_extra:
        from sdr_b200 import workloads
        cpu = not args.no_cpu
        rec, s, sdf = frame_record(workloads.plain_parametric(), "parametric_0p8mm", cpu, args.cpu_budget)
        s.close()
        line.update(rec)
        w = workloads.real_cavity(seed=2)
        rec, s, sdf = frame_record(w, "cavity_0p5mm", cpu, args.cpu_budget)
        line.update(rec)
        line.update(render_bench(s, w, sdf, cpu=cpu))
        s.close()
        if not args.no_batch and args.batch_scenes > 0:
            line.update(batch_bench(args.batch_scenes, args.batch_cfl))
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
