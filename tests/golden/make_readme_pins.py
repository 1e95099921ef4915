"""Regenerate readme_pins.json: the oracle run on the reference's two README scenes.

Reads the reference checkout named by $SDR_REFERENCE (required) at generation
time only; the committed JSON is what the tests read. The pinned
README figures (uselessgoddess/sdr README.md:58-61 and 146-151):
  examples/scene.toml          peak fill 19.9 %, peak coverage 59.1 %,
                               peak membrane 1099.3 mmHg (146558 Pa),
                               mean membrane 3.3 mmHg (436 Pa), drained 8.11 ml of 10.0
  examples/maxillary_real.toml fill 44.9 %, 92 % of fluid in the lower half (along gravity)
Usage: python tests/golden/make_readme_pins.py [scene|maxillary] [threads] [variant]

variant (optional) reruns the scene perturbed, to measure how far its chaotic
summary moves on its own: "f32" rounds the particle state to f32 after every
substep (the device's storage precision), "seed" starts the emission stream
from another seed (0x9e3779b97f4a7c15). The result goes to the scene's
"variants" entry. "noredist" and "nosource" switch one physics option off
(Solver::redistribute, solver.rs:454-557; the volume source, solver.rs:392-423)
to see which of them moves the summary towards the README's figures.
"walls" reruns the scene unperturbed, records every cell holding a particle at
a frame end, and reports the peak wall coverage under other definitions of
the wall (metrics.rs:133-170 is the first; the rest are what an earlier
revision might have used): no domain-edge cells, contact through any of the
26 neighbours, and a lining two cells deep; and the reference wall's
coverage when only every 2nd, 3rd, 4th or 6th frame end is sampled (washed
cells are marked only at frame ends, metrics.rs:196-204).
"""
import dataclasses
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import numpy as np  # noqa: E402

import oracle  # noqa: E402
from sdr_b200 import scene as sc  # noqa: E402
from tests.helpers import cavity_volume, oracle_sdf, oracle_solver  # noqa: E402

REF = os.environ.get("SDR_REFERENCE")


VARIANT_SEED = 0x9E3779B97F4A7C15


def run(name: str, threads: int, variant: str = ""):
    if not REF:
        raise SystemExit("set SDR_REFERENCE to the reference checkout (the directory holding examples/)")
    oracle.set_threads(threads)
    path = os.path.join(REF, "examples", f"{name}.toml")
    cfg = sc.SceneConfig.from_toml_file(path)
    if cfg.sinus["mesh"] is not None:
        cfg.sinus["mesh"] = os.path.join(REF, cfg.sinus["mesh"])
    res = cfg.resolve()
    if variant == "noredist":
        res = dataclasses.replace(res, fluid=dataclasses.replace(res.fluid, redistribute=False))
    elif variant == "nosource":
        res = dataclasses.replace(res, fluid=dataclasses.replace(res.fluid, volume_stiffness=0.0))
    tris = None if res.sinus is not None else sc.load_mesh(res.mesh_path) * sc.MM
    t0 = time.time()
    sdf = oracle_sdf(res, tris)
    s = oracle_solver(res, sdf)
    vol = cavity_volume(res, tris)
    m = oracle.Metrics(s, vol)
    if variant == "seed":
        sc0 = s.scalars()
        s.set_scalars(sc0["time"], sc0["emit_accum"], sc0["steps"], sc0["drained"], VARIANT_SEED)
    frames = []
    visited = None
    per_frame = []
    if variant == "walls":
        nx_, ny_, nz_ = s.grid[0]
        visited = np.zeros(nx_ * ny_ * nz_, dtype=bool)
    for f in range(res.frames):
        if variant == "f32":  # Solver::step (solver.rs:237-259) with the state rounded after every substep
            remaining, floor, taken = res.frame_dt, res.frame_dt / 512, 0
            while remaining > 1e-12:
                sub = min(max(s.cfl_dt(), floor), remaining)
                s.substep(sub)
                p, v = s.particles()
                s.set_particles(p.astype(np.float32).astype(np.float64), v.astype(np.float32).astype(np.float64))
                remaining -= sub
                taken += 1
        else:
            s.step(res.frame_dt)
        r = m.record(s, f)
        if visited is not None:
            occ = _occupied(s)
            visited[occ] = True
            per_frame.append(np.unique(occ))
        r["substeps"] = s.scalars()["last_substeps"] if variant != "f32" else taken
        frames.append(r)
        print(name, f, r["time_s"], r["particles"], r["fill_fraction"], r["pcg_iters"], r["substeps"],
              f"{time.time() - t0:.0f}s", flush=True)
    if visited is not None:
        walls = _wall_definitions(s)
        cov = {k: float((visited & wm).sum() / max(int(wm.sum()), 1)) for k, wm in walls.items()}
        cov["counts"] = {k: int(wm.sum()) for k, wm in walls.items()}
        ref = walls["reference"]
        for every in (2, 3, 4, 6):
            sub = np.zeros_like(visited)
            for f in range(every - 1, len(per_frame), every):
                sub[per_frame[f]] = True
            cov[f"reference_every_{every}_frames"] = float((sub & ref).sum() / max(int(ref.sum()), 1))
    out = {"scene": f"examples/{name}.toml", "summary": m.summary(), "frames": frames,
           "cavity_volume_m3": vol, "grid": list(s.grid[0]), "wall_seconds": time.time() - t0,
           "threads": threads}
    if visited is not None:
        out["coverage_by_wall_definition"] = cov
    pos, _ = s.particles()
    if len(pos):
        g = np.asarray(res.fluid.gravity, dtype=np.float64)
        gd = g / np.linalg.norm(g)
        depth = pos @ gd  # larger = lower along gravity
        mn, mx = sdf.bounds()
        # cavity extent along gravity from the SDF's interior nodes
        nz, ny, nx = sdf.data.shape
        kk, jj, ii = np.nonzero(sdf.data < 0)
        pts = np.stack([sdf.origin[0] + ii * sdf.dx, sdf.origin[1] + jj * sdf.dx, sdf.origin[2] + kk * sdf.dx], 1)
        d = pts @ gd
        mid = 0.5 * (d.min() + d.max())
        out["fraction_lower_half"] = float(np.mean(depth > mid))
    return out


def _occupied(s):
    """Cells holding a particle (MetricsCollector::cell_index, metrics.rs:434-445)."""
    (nx, ny, nz), origin, dx = s.grid[0], np.asarray(s.grid[1], dtype=np.float64), s.grid[2]
    p, _ = s.particles()
    if not len(p):
        return np.zeros(0, dtype=np.int64)
    l = (p - origin) / dx
    ok = np.all(l >= 0.0, axis=1)
    ijk = np.floor(l[ok]).astype(np.int64)
    ok2 = (ijk[:, 0] < nx) & (ijk[:, 1] < ny) & (ijk[:, 2] < nz)
    ijk = ijk[ok2]
    return (ijk[:, 2] * ny + ijk[:, 1]) * nx + ijk[:, 0]


def _wall_definitions(s):
    """Wall masks from the cavity cells: the reference's (an inside cell with a
    non-inside face neighbour, the domain edge counting as non-inside) and the
    alternatives described in the module docstring."""
    nx, ny, nz = s.grid[0]
    inside = s.cavity_mask().reshape(nz, ny, nx).astype(bool)

    def shifted(a, d, axis, fill):
        out = np.full_like(a, fill)
        src = [slice(None)] * 3
        dst = [slice(None)] * 3
        if d > 0:
            src[axis], dst[axis] = slice(d, None), slice(None, -d)
        else:
            src[axis], dst[axis] = slice(None, d), slice(-d, None)
        out[tuple(dst)] = a[tuple(src)]
        return out

    def face_touch(edge_fill):
        t = np.zeros_like(inside)
        for axis in range(3):
            for d in (-1, 1):
                t |= ~shifted(inside, d, axis, not edge_fill)
        return inside & t

    ref = face_touch(True)
    no_edge = face_touch(False)
    t26 = np.zeros_like(inside)
    for dk in (-1, 0, 1):
        for dj in (-1, 0, 1):
            for di in (-1, 0, 1):
                if dk == dj == di == 0:
                    continue
                a = inside
                for axis, d in ((0, dk), (1, dj), (2, di)):
                    if d:
                        a = shifted(a, d, axis, False)
                t26 |= ~a
    all26 = inside & t26
    second = np.zeros_like(inside)
    for axis in range(3):
        for d in (-1, 1):
            second |= shifted(ref, d, axis, False)
    two_deep = ref | (inside & second)
    return {"reference": ref.reshape(-1), "no_domain_edge": no_edge.reshape(-1), "contact_26": all26.reshape(-1),
            "two_cells_deep": two_deep.reshape(-1)}


if __name__ == "__main__":
    which = sys.argv[1] if len(sys.argv) > 1 else "scene"
    threads = int(sys.argv[2]) if len(sys.argv) > 2 else 4
    variant = sys.argv[3] if len(sys.argv) > 3 else ""
    res = run(which, threads, variant)
    dst = os.path.join(HERE, "readme_pins.json")
    data = json.load(open(dst)) if os.path.exists(dst) else {}
    if variant:
        entry = {"summary": res["summary"], "wall_seconds": res["wall_seconds"]}
        if "coverage_by_wall_definition" in res:
            entry["coverage_by_wall_definition"] = res["coverage_by_wall_definition"]
        data[which].setdefault("variants", {})[variant] = entry
    else:
        data[which] = res
    with open(dst, "w") as f:
        json.dump(data, f, indent=1)
    print(json.dumps(res["summary"], indent=1))
