"""Many scenes on one GPU: every scene's result is the same alone, one after
another, and in a concurrent mix (batch or server), and equals the plain
single-solver path. Scenes are small (the smoke sinus at 2 mm, 2 frames)."""
import numpy as np
import pytest

from sdr_b200 import _lib, scene as sc
from sdr_b200.serving import SceneSpec, Server, footprint, run_batch
from tests.gpu_common import SMOKE_TOML, record

pytestmark = pytest.mark.gpu

FIELDS = ("frames", "final_time_s", "peak_fill_fraction", "final_fill_fraction", "peak_wall_coverage",
          "final_wall_coverage", "peak_membrane_pressure_pa", "mean_membrane_pressure_pa", "peak_pressure_pa",
          "membrane_artifacts_total", "total_drained_ml", "injected_ml", "mass_balance")


def _specs(flows=(3.0, 5.0, 7.0), frames=2):
    from sdr_b200.solver import build_sdf, cavity_volume
    base = sc.SceneConfig.from_toml_str(SMOKE_TOML).resolve()
    sdf = build_sdf(base)
    vol = cavity_volume(base, sdf)
    out = []
    for f in flows:
        n = base.needle
        needle = sc.Needle(tip=n.tip, axis=n.axis, radius=n.radius, flow_rate=f * sc.ML_PER_S,
                           inject_until=n.inject_until)
        out.append(SceneSpec(sdf=sdf, sim_dx=base.sim_dx, fluid=base.fluid, needle=needle, solve=base.solve,
                             cavity_volume=vol, frame_dt=base.frame_dt, frames=frames, outlet=base.outlet))
    return out


def _same(a: dict, b: dict):
    for k in FIELDS:
        assert a[k] == b[k], (k, a[k], b[k])


def _plain(spec: SceneSpec) -> dict:
    """The single-scene API path: Solver + MetricsCollector, frame by frame."""
    from sdr_b200.solver import MetricsCollector, Solver
    s = Solver(spec.sdf, spec.sim_dx, spec.fluid, spec.needle)
    s.solve = spec.solve
    s.outlet = spec.outlet
    m = MetricsCollector(s, spec.cavity_volume)
    for f in range(spec.frames):
        s.step(spec.frame_dt)
        m.record(s, f)
    return m.summary()


def test_batch_same_alone_sequential_and_concurrent():
    specs = _specs()
    seq = run_batch(specs, concurrency=1)
    mix = run_batch(specs, concurrency=0)
    assert all(r.status == _lib.SDR_OK for r in seq + mix), [r.error for r in seq + mix]
    for a, b in zip(seq, mix):
        _same(a.summary, b.summary)
        assert a.stats["particles"] == b.stats["particles"] and a.stats["steps"] == b.stats["steps"]
    alone = _plain(specs[1])
    _same(alone, mix[1].summary)
    record("batch", {"seconds_sequential": sum(r.seconds for r in seq), "seconds_each_in_mix": [r.seconds for r in mix],
                     "fill": [r.summary["final_fill_fraction"] for r in mix]})


def test_server_continuous_batching_matches_batch():
    specs = _specs(flows=(2.0, 3.0, 4.0, 5.0, 6.0))
    ref = run_batch(specs, concurrency=1)
    with Server(budget_bytes=64 << 30, max_active=2) as srv:
        tickets = [srv.submit(s) for s in specs[:3]]
        more = [srv.submit(s) for s in specs[3:]]  # arrive while the first ones run
        res = srv.wait(tickets + more, timeout=600)
        st = srv.stats()
    assert all(r.status == _lib.REQ_DONE for r in res), [r.error for r in res]
    for a, b in zip(ref, res):
        _same(a.summary, b.summary)
        assert b.seconds > 0.0
    assert st["completed"] == 5 and st["failed"] == 0 and 1 <= st["peak_active"] <= 2
    assert st["active"] == 0 and st["bytes_in_use"] == 0
    record("server", {"stats": st, "time_to_summary": [r.seconds for r in res]})


def test_server_budget_admits_one_at_a_time():
    specs = _specs(flows=(3.0, 6.0))
    fp = max(footprint(s) for s in specs)
    with Server(budget_bytes=int(fp * 1.5), max_active=4) as srv:
        res = srv.wait([srv.submit(s) for s in specs], timeout=600)
        st = srv.stats()
    assert all(r.status == _lib.REQ_DONE for r in res)
    assert st["peak_active"] == 1 and st["peak_bytes"] <= int(fp * 1.5)


def test_metrics_outlive_solver_and_growth_matches_preallocated():
    """Device buffers are released in stream order: a collector destroyed after
    its solver still answers its summary, and particle arrays that grow mid-run
    (a stream-ordered copy into the larger arrays) give the same scene as
    arrays sized for the whole run up front."""
    from sdr_b200.solver import MetricsCollector, Solver
    spec = _specs(flows=(8.0,), frames=4)[0]

    def run(max_particles):
        s = Solver(spec.sdf, spec.sim_dx, spec.fluid, spec.needle, max_particles=max_particles)
        s.solve = spec.solve
        s.outlet = spec.outlet
        m = MetricsCollector(s, spec.cavity_volume)
        for f in range(spec.frames):
            s.step(spec.frame_dt)
            m.record(s, f)
        n = len(s)
        s.close()  # the solver goes first
        out = m.summary()
        m.close()
        return out, n

    small, n_small = run(256)  # grows several times while the jet fills the cavity
    big, n_big = run(1 << 20)
    assert n_small > 4 * 256 and n_small == n_big
    _same(small, big)


def test_packed_batch_one_launch_per_operation_same_results():
    """sdr_batch_run_packed: every packed step advances all live scenes by one
    substep with one launch per substep operation (ragged offset table,
    persistent grid). The scenes - uneven flows and so uneven particle counts,
    substep counts and PCG iterations - give the same summaries, stats and
    particle counts bit for bit as one after another on their own solvers, and
    the launches are those of the busiest scene, not of all scenes."""
    specs = _specs(flows=(2.0, 4.0, 6.0, 8.0), frames=3)
    seq = run_batch(specs, concurrency=1)
    cnt = {}
    packed = run_batch(specs, packed=True, counters=cnt)
    assert all(r.status == _lib.SDR_OK for r in seq + packed), [r.error for r in seq + packed]
    for a, b in zip(seq, packed):
        _same(a.summary, b.summary)
        for k in ("particles", "steps", "drained", "emitted", "culled", "particle_substeps", "last_pcg_iters"):
            assert a.stats[k] == b.stats[k], (k, a.stats[k], b.stats[k])
    subs = [r.stats["substeps_total"] for r in seq]
    assert cnt["steps"] == max(subs)
    per_step = cnt["launches"] / cnt["steps"]
    record("packed_batch", {"counters": cnt, "launches_per_packed_step": per_step, "substeps": subs,
                            "seconds_sequential": sum(r.seconds for r in seq),
                            "seconds_packed": max(r.seconds for r in packed)})
    assert per_step < 90  # one launch per operation, whatever the number of scenes
    assert cnt["graph_captures"] < cnt["steps"] / 4  # the packed step's graph is replayed


def test_packed_server_continuous_batching_matches_batch():
    """The request loop with one packed engine: requests that arrive while
    others run join the packed steps as slots free up; each result equals its
    scene run alone."""
    specs = _specs(flows=(2.0, 3.0, 4.0, 5.0, 6.0))
    ref = run_batch(specs, concurrency=1)
    with Server(budget_bytes=64 << 30, max_active=3, packed=True) as srv:
        tickets = [srv.submit(s) for s in specs[:2]]
        more = [srv.submit(s) for s in specs[2:]]
        res = srv.wait(tickets + more, timeout=600)
        st = srv.stats()
    assert all(r.status == _lib.REQ_DONE for r in res), [r.error for r in res]
    for a, b in zip(ref, res):
        _same(a.summary, b.summary)
    assert st["completed"] == 5 and st["failed"] == 0 and 1 <= st["peak_active"] <= 3
    assert st["active"] == 0 and st["bytes_in_use"] == 0
    record("packed_server", {"stats": st, "time_to_summary": [r.seconds for r in res]})
