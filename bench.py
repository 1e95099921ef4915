#!/usr/bin/env python
"""Benchmark: particle-substeps/s of the FLIP/PIC substep on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl sdr|reference] [--workload real_cavity]

A step is one output frame (Solver::step(frame_dt), all its CFL substeps) of
the workload. W frames warm up, K frames are timed. ``value`` is device time
(CUDA events on the solver stream, summed over the timed frames, max over
ranks); ``e2e`` is the same frames timed on the host around the public call
plus the per-frame read-back of particle positions (host buffers). Between
timed frames a 256 MiB buffer is written to flush L2.

Multi-GPU runs are independent scene replicas (one per rank, different cavity
seeds): no collective on the data path; a barrier and a max-reduce of the
timings use torch.distributed.

``--impl reference`` times the CPU restatement of the reference solver
(oracle/, the reference Rust cannot be built here) on the host cores: W
frames from t = 0 to reach the timed window, then K bounded samples.

``batched`` and ``served`` (one GPU): a bounded sample of the batched scene
family (seeded perturbed-ellipsoid cavities, grids log-uniform in 32^3..96^3
cells, random needle tilt, flow and dose). Each of ``--batch-scenes`` scenes
runs one frame of ``--batch-cfl`` jet-CFL steps (frame_dt = n * dx / jet
speed), so that per-scene work varies with the grid alone instead of being
dominated by the finest, fastest jets. The scenes run one after another
through the public calls (the plain path), all at once (sdr_batch_run), and as
Poisson arrivals into the request server (sdr_server_*, 150 GB admission
budget) with p50/p99 time-to-summary.

``render``: preview images (render_slice, 600 px) of the final state, the
slice through the needle tip and the gravity projection, timed through the
public call, beside the oracle drawing the same state.

``large`` (one GPU): the 0.2 mm parametric cavity (207 x 217 x 161 cells)
with a pre-seeded pool of 9.5 M particles at rest, ``--large-substeps``
substeps at the fixed jet CFL step after ``--large-warmup``, device-timed;
the oracle times one substep of the identical state.
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

# Algorithmic bytes of the pressure solve (the dominant kernel, k_pcg), f64
# vectors in wavefront order: per fluid cell and PCG iteration, and per fluid
# cell once per solve (factorisation, first preconditioner application, setup).
PCG_BYTES_PER_CELL_ITER = 233
PCG_BYTES_PER_CELL_SOLVE = 190


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


def oracle_for(w, sdf):
    import oracle
    from tests.helpers import oracle_solver
    osdf = oracle.SdfGrid(tuple(sdf.origin), sdf.dx, sdf.data)
    return oracle_solver(w.res, osdf)


def cpu_sample(orc, budget_s: float, max_substeps: int):
    """Run the oracle for a bounded sample; returns (particle_substeps, seconds, substeps)."""
    t0 = time.perf_counter()
    ps = sub = 0
    while sub < max_substeps and time.perf_counter() - t0 < budget_s:
        dt = orc.cfl_dt()
        ps += len(orc) + 0
        orc.substep(dt)
        sub += 1
    return ps, time.perf_counter() - t0, sub


def run_reference(args):
    """CPU restatement of the reference (all host threads), same workload and metric."""
    import oracle
    from sdr_b200 import workloads
    from sdr_b200.solver import Sdf
    w = workloads.WORKLOADS[args.workload]()
    # The reference arm builds its SDF with the oracle's own winding-number/implicit code.
    if w.res.sinus is not None:
        osdf = oracle.sdf_from_sinus(w.res.sinus, w.res.sdf_origin, w.res.sdf_dx, w.res.sdf_dims)
    else:
        osdf = oracle.sdf_from_mesh(w.tris, w.res.sdf_dx, w.res.mesh_padding)
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    from tests.helpers import oracle_solver
    orc = oracle_solver(w.res, osdf)
    for _ in range(args.warmup):
        orc.step(w.res.frame_dt)
    ps_tot = 0
    t_tot = 0.0
    subs = 0
    for _ in range(args.steps):
        ps, t, sub = cpu_sample(orc, budget_s=args.ref_budget, max_substeps=args.ref_substeps)
        ps_tot += ps
        t_tot += t
        subs += sub
    v = ps_tot / t_tot if t_tot > 0 else 0.0
    sample = (f"{args.warmup} frames from t=0 (untimed), then {args.steps} samples of up to "
              f"{args.ref_substeps} substeps ({subs} substeps, {ps_tot} particle-substeps)")
    line = {"metric": "particle-substeps/s", "value": v, "unit": "particle-substeps/s", "impl": "reference",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_tot / max(args.steps, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": w.name, **(w.describe or {})},
            "cpu_baseline": {"value": v, "unit": "particle-substeps/s", "cores": threads, "kind": "port",
                             "sample": sample + "; C++ restatement of the reference solver (Rust not buildable)"},
            "e2e": {"value": v, "unit": "particle-substeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def batch_bench(n_scenes: int, cfl_steps: int, seed0: int = 100) -> dict:
    """Plain (one scene after another), batched and served runs of the same scenes."""
    import math
    import random
    from sdr_b200 import _lib, workloads
    from sdr_b200.serving import Server, run_batch
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
    ok = all(r.status == _lib.SDR_OK for r in plain + mix)
    same = ok and all(a.summary == b.summary for a, b in zip(plain, mix))
    ps = sum(r.stats["particle_substeps"] for r in mix) if ok else 0
    subs = sum(r.stats["substeps_total"] for r in mix) if ok else 0
    rate = 0.8 * n_scenes / t_mix  # arrivals at 80 % of the batched throughput
    rng = random.Random(seed0)
    with Server(budget_bytes=150 << 30, max_active=n_scenes) as srv:
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
    lat = sorted(r.seconds for r in res)
    served_same = ok and all(r.summary == b.summary for r, b in zip(res, mix))

    def pct(q):
        return lat[min(len(lat) - 1, int(round(q * (len(lat) - 1))))]
    sample = (f"{n_scenes} scenes of the batched family (seeds {seed0}..{seed0 + n_scenes - 1}), each one frame "
              f"of {cfl_steps} jet-CFL steps from t = 0; SDFs built on the device in {build_s:.1f} s")
    return {
        "batched": {"scenes": n_scenes, "cfl_steps_per_scene": cfl_steps, "sample": sample,
                    "plain_scenes_per_s": n_scenes / t_plain, "batched_scenes_per_s": n_scenes / t_mix,
                    "speedup": t_plain / t_mix, "plain_s": t_plain, "batched_s": t_mix,
                    "particle_substeps_per_s": ps / t_mix, "substeps": subs, "results_identical": same},
        "served": {"arrivals": "poisson", "rate_per_s": rate, "scenes_per_s": n_scenes / t_srv,
                   "p50_time_to_summary_s": pct(0.5), "p99_time_to_summary_s": pct(0.99),
                   "peak_active": sst["peak_active"], "peak_bytes": sst["peak_bytes"],
                   "budget_bytes": 150 << 30, "results_identical": served_same},
    }


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


def large_bench(n_sub: int, warm: int, cpu: bool) -> dict:
    """The 0.2 mm parametric cavity (207 x 217 x 161 cells) with a pre-seeded
    pool: the deepest cavity cells filled at 8 particles per cell with
    hash_jitter offsets, at rest (9.5 M particles, the cavity holds fewer than
    the 30 M asked for), then substeps at the fixed jet CFL step. Inputs are far
    larger than L2. The oracle times one substep of the identical state."""
    import numpy as np
    from sdr_b200 import workloads
    w = workloads.large_parametric()
    t0 = time.perf_counter()
    solver, sdf, vol = workloads.build_gpu(w, max_particles=12_000_000)
    pos, vel = workloads.preseed_pool(solver, 30_000_000)
    pos = pos.astype(np.float32).astype(np.float64)  # the stored (f32) state, shared with the oracle
    solver.set_particles(pos, vel)
    setup_s = time.perf_counter() - t0
    jet = solver.needle.flow_rate / (np.pi * solver.needle.radius ** 2)
    dt = solver.dx / jet
    solver.set_profiling(True)
    for _ in range(warm):
        solver.substep(dt)
    solver.reset_profile()
    st0 = solver.stats()
    t0 = time.perf_counter()
    for _ in range(n_sub):
        solver.substep(dt)
    wall = time.perf_counter() - t0
    st1 = solver.stats()
    prof = solver.profile()
    dev_ms = st1.device_ms - st0.device_ms
    ps = st1.particle_substeps - st0.particle_substeps
    out = {"workload": "large_parametric, pre-seeded pool", "grid": [st1.nx, st1.ny, st1.nz],
           "particles": int(len(pos)), "dt_s": dt, "warmup_substeps": warm, "substeps": n_sub,
           "particle_substeps_per_s": ps / (dev_ms / 1e3), "wall_particle_substeps_per_s": ps / wall,
           "ms_per_substep": dev_ms / n_sub, "setup_s": setup_s,
           "phase_ms": {k: round(v, 3) for k, v in prof.items() if k.endswith("_ms")},
           "pcg": {"mean_iters": prof["pcg_cell_iters"] / max(prof["fluid_cells"], 1),
                   "mean_fluid_cells": prof["fluid_cells"] / max(prof["pcg_launches"], 1),
                   "cluster_launches": prof["pcg_cluster_launches"]},
           "redistribution": {"candidates": prof["redist_candidates"], "sweeps": prof["redist_sweeps"],
                              "long_sweeps": prof["redist_long_sweeps"]}}
    solver.close()
    if cpu:
        import oracle
        orc = oracle_for(w, sdf)
        orc.set_particles(pos, vel)
        threads = os.cpu_count() or 1
        oracle.set_threads(threads)
        t0 = time.perf_counter()
        orc.substep(dt)
        ct = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": len(pos) / ct, "unit": "particle-substeps/s", "cores": threads,
                               "kind": "port", "sample": f"one substep of the pre-seeded state ({ct:.1f} s); "
                                                         "C++ restatement of the reference solver, f64"}
    return {"large": out}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="sdr", choices=["sdr", "reference"])
    ap.add_argument("--workload", default="real_cavity")
    ap.add_argument("--cpu-budget", type=float, default=15.0, help="seconds of oracle time for cpu_baseline")
    ap.add_argument("--ref-budget", type=float, default=20.0)
    ap.add_argument("--ref-substeps", type=int, default=20)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--batch-scenes", type=int, default=48)
    ap.add_argument("--batch-cfl", type=int, default=150)
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-large", action="store_true")
    ap.add_argument("--large-substeps", type=int, default=5)
    ap.add_argument("--large-warmup", type=int, default=3)
    args = ap.parse_args()
    rank, world, local = dist_env()

    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return

    import numpy as np
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from sdr_b200 import _lib, workloads

    w = workloads.WORKLOADS[args.workload]() if args.workload != "real_cavity" else workloads.real_cavity(seed=2 + rank)
    solver, sdf, vol = workloads.build_gpu(w)
    solver.set_profiling(True)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for _ in range(args.warmup):
        solver.step(w.res.frame_dt)
    solver.reset_profile()
    launches0 = _lib.load().sdr_kernel_launch_count()
    clk = Clocks(local)
    dev_ms = 0.0
    wall = 0.0
    ps = 0
    h2d = 0
    d2h = 0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        st0 = solver.stats()
        t0 = time.perf_counter()
        solver.step(w.res.frame_dt)          # public API: host emission uploads inside
        pos, _ = solver.particles_f32()      # per-frame result read-back (positions)
        t1 = time.perf_counter()
        st1 = solver.stats()
        dev_ms += st1.device_ms - st0.device_ms
        wall += t1 - t0
        ps += st1.particle_substeps - st0.particle_substeps
        h2d += (st1.emitted - st0.emitted) * 32 + (st1.substeps_total - st0.substeps_total) * 4
        d2h += pos.nbytes * 2 + (st1.substeps_total - st0.substeps_total) * 96
    torch.cuda.synchronize()
    clocks = clk.stop()
    launches = _lib.load().sdr_kernel_launch_count() - launches0
    prof = solver.profile()
    # One more frame, not timed, with the section timers inside the pressure
    # solve switched on (they sit on its critical path, so the timed frames
    # run without them): the per-section cycle split of k_pcg.
    solver.reset_profile()
    solver.set_profiling(True, kernel_timers=True)
    solver.step(w.res.frame_dt)
    diag = solver.profile()
    solver.set_profiling(False)
    if world > 1:
        dev_ms, wall, ps = reduce_over_ranks(dev_ms, wall, ps, "cuda")
    value = ps / (dev_ms / 1e3)
    e2e = ps / wall
    hbm, peak_kind = peaks()
    pcg_launch_ms = prof["pcg_ms"] / max(prof["pcg_launches"], 1)
    pcg_bytes = (PCG_BYTES_PER_CELL_ITER * prof["pcg_cell_iters"] + PCG_BYTES_PER_CELL_SOLVE * prof["fluid_cells"]) / max(prof["pcg_launches"], 1)
    achieved = pcg_bytes / (pcg_launch_ms / 1e3) / 1e9 if pcg_launch_ms > 0 else 0.0
    st = solver.stats()
    sub_bytes = substep_bytes(prof["particles"], prof["substeps"], int(st.nx * st.ny * st.nz),
                              int(sdf.data.size), prof["pcg_cell_iters"])
    sub_gbs = sub_bytes / (dev_ms / 1e3) / 1e9 if dev_ms > 0 else 0.0  # rank 0's substeps, rank 0's time at N = 1
    line = {"metric": "particle-substeps/s", "value": value, "unit": "particle-substeps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic",
            "config": {"workload": w.name, **(w.describe or {}), "grid": [st.nx, st.ny, st.nz],
                       "particles_end": int(st.particles), "substeps": int(prof["substeps"]),
                       "l2": "256 MiB buffer written between timed frames", "replicas": world},
            "e2e": {"value": e2e, "unit": "particle-substeps/s", "h2d_bytes_per_step": int(h2d / args.steps),
                    "d2h_bytes_per_step": int(d2h / args.steps)},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "roofline": {"bound": "hbm", "kernel": "k_pcg", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "peak_kind": peak_kind, "traffic": None,
                         "bytes_per_launch": pcg_bytes, "ms_per_launch": pcg_launch_ms},
            "substep_roofline": ({"bound": "hbm", "achieved": sub_gbs, "peak": hbm, "unit": "GB/s",
                                  "frac": sub_gbs / hbm, "peak_kind": peak_kind,
                                  "bytes_per_substep": sub_bytes / max(prof["substeps"], 1),
                                  "bytes": "112 P + 92 C + 4 S + 83 N_f iters per substep"}
                                 if world == 1 else None),
            "phase_ms": {k: round(v, 3) for k, v in prof.items() if k.endswith("_ms")},
            "pcg_section_cycles": {k: v for k, v in zip(
                ["mic_build", "sweeps", "unused", "matvec", "dots", "axpy_norm", "direction", "setup_exit",
                 "lvl_stage_wait", "lvl_compute", "lvl_barrier", "lvl_count", "sum_sweep_width", "sum_level_range",
                 "solves"], diag["pcg_section_cycles"]) if k not in ("unused", "lvl_stage_wait")},
            "pcg_section_cycles_frame": "one untimed frame after the timed ones, in-kernel section timers on",
            "pcg": {"launches": prof["pcg_launches"], "mean_iters": prof["pcg_cell_iters"] / max(prof["fluid_cells"], 1),
                    "mean_fluid_cells": prof["fluid_cells"] / max(prof["pcg_launches"], 1)},
            "redistribution": {"candidates": prof["redist_candidates"], "sweeps": prof["redist_sweeps"],
                               "long_sweeps": prof["redist_long_sweeps"]}}
    if rank == 0 and not args.no_cpu:
        orc = oracle_for(w, sdf)
        pos, vel = solver.particles()
        orc.set_particles(pos, vel)
        s = solver.stats()
        orc.set_scalars(s.time, s.emit_accum, s.steps, s.drained, s.rng_state)
        import oracle
        threads = os.cpu_count() or 1
        oracle.set_threads(threads)
        cps, ct, csub = cpu_sample(orc, budget_s=args.cpu_budget, max_substeps=10 ** 9)
        line["cpu_baseline"] = {"value": cps / ct, "unit": "particle-substeps/s", "cores": threads, "kind": "port",
                                "sample": f"{csub} substeps from the GPU state one frame after the timed frames "
                                          f"({cps} particle-substeps, {ct:.1f} s); C++ restatement of the "
                                          "reference solver, f64, rayon-parallel parts on all host threads"}
    if rank == 0 and world == 1:
        line.update(render_bench(solver, w, sdf, cpu=not args.no_cpu))
    if rank == 0 and world == 1 and not args.no_batch and args.batch_scenes > 0:
        solver.close()
        line.update(batch_bench(args.batch_scenes, args.batch_cfl))
    if rank == 0 and world == 1 and not args.no_large:
        solver.close()  # idempotent
        line.update(large_bench(args.large_substeps, args.large_warmup, cpu=not args.no_cpu))
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
