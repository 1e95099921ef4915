"""The oracle against the reference's own known-answer and invariant tests.

Each test restates one of uselessgoddess/sdr's in-file unit tests (cited) and
checks the CPU oracle with the same values and tolerances, pinning the
restatement before it is used to check the CUDA path.
"""
import math

import numpy as np
import pytest

import oracle
from sdr_b200 import scene as sc
from tests.helpers import cavity_volume, oracle_solver


# ---------------------------------------------------------------- sdf.rs
def test_point_triangle_distance_basic():  # sdf.rs:338-348
    a, b, c = (0, 0, 0), (1, 0, 0), (0, 1, 0)
    assert abs(oracle.point_triangle_distance_sq((0.25, 0.25, 2.0), a, b, c) - 4.0) < 1e-12
    assert abs(oracle.point_triangle_distance_sq((-1.0, -1.0, 0.0), a, b, c) - 2.0) < 1e-12


def box_tris():
    v = np.array([(-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1), (-1, -1, 1), (1, -1, 1), (1, 1, 1), (-1, 1, 1)],
                 dtype=np.float64)
    f = [(0, 3, 2), (0, 2, 1), (4, 5, 6), (4, 6, 7), (0, 1, 5), (0, 5, 4), (3, 7, 6), (3, 6, 2), (0, 4, 7), (0, 7, 3),
         (1, 2, 6), (1, 6, 5)]
    return np.array([np.concatenate([v[i], v[j], v[k]]) for i, j, k in f])


def test_winding_sign_for_box():  # sdf.rs:298-335
    t = box_tris()
    assert abs(oracle.signed_distance_to_mesh((0, 0, 0), t) - (-1.0)) < 1e-9
    d_out = oracle.signed_distance_to_mesh((3, 0, 0), t)
    assert d_out > 0 and abs(d_out - 2.0) < 1e-9


def test_sphere_sdf_matches_analytic():  # sdf.rs:280-295
    sdf = oracle.sdf_from_fn((-2.0, -2.0, -2.0), 0.2, (21, 21, 21), lambda p: float(np.linalg.norm(p)) - 1.0)
    assert abs(sdf.sample((0, 0, 0)) - (-1.0)) < 1e-9
    assert abs(sdf.sample((1.5, 0, 0)) - 0.5) < 1e-9
    g = sdf.gradient((1.5, 0, 0))
    assert 0.9 < g[0] < 1.1
    assert sdf.sample((0, 0, 0)) < 0 and not sdf.sample((2.0, 0, 0)) < 0


# ---------------------------------------------------------------- solver.rs
def test_jet_speed_from_flow_rate():  # solver.rs:1046-1056
    n = sc.Needle(tip=(0, 0, 0), axis=(0, 1, 0), radius=0.001, flow_rate=1e-6)
    assert abs(n.jet_speed() - 1.0 / math.pi) < 1e-9


def box_solver(ppc=8):  # solver.rs:1170-1189
    dx = 0.002
    a = 0.012
    sdf = oracle.sdf_from_fn((-0.016, -0.016, -0.016), dx, (16, 16, 16),
                             lambda p: max(abs(p[0]) - a, abs(p[1]) - a, abs(p[2]) - a))
    return oracle.Solver(sdf, dx, oracle.Fluid(particles_per_cell=ppc),
                         oracle.Needle((0.0, 0.010, 0.0), (0.0, -1.0, 0.0), 0.0006, 5.0e-6))


def pack_one_cell(s, cell, n):  # solver.rs:1192-1202
    (nx, ny, nz), origin, dx = s.grid
    center = origin + (np.array(cell) + 0.5) * dx
    pos = np.array([center + oracle.hash_jitter(i) * dx for i in range(n)])
    s.set_particles(pos, np.zeros_like(pos))
    return center


def count_at(s, ijk):
    (nx, ny, nz), origin, dx = s.grid
    pos, _ = s.particles()
    l = (pos - origin) / dx
    c = np.floor(l).astype(int)
    return int(np.sum(np.all(c == np.array(ijk), axis=1)))


def test_redistribution_drains_surplus_downhill():  # solver.rs:1212-1243
    s = box_solver()
    cap, surplus = 8, 4
    pack_one_cell(s, (8, 8, 8), cap + surplus)
    s.phase(oracle.PHASE_REDISTRIBUTE)
    assert len(s) == cap + surplus
    assert count_at(s, (8, 8, 8)) == cap
    assert count_at(s, (8, 7, 8)) == surplus
    assert count_at(s, (8, 9, 8)) == 0


def test_redistribution_relieves_overpacked_cell_and_conserves_mass():  # solver.rs:1251-1335
    N = 100
    s = box_solver()
    center = pack_one_cell(s, (8, 8, 8), N)
    assert s.sdf.sample(center) < 0
    assert s.max_particles_per_cell() == N
    s.phase(oracle.PHASE_REDISTRIBUTE)
    assert len(s) == N
    assert s.max_particles_per_cell() < N
    (nx, ny, nz), origin, dx = s.grid
    pos, _ = s.particles()
    c = np.floor((pos - origin) / dx).astype(int)
    keys = (c[:, 2] * ny + c[:, 1]) * nx + c[:, 0]
    counts = np.bincount(keys, minlength=nx * ny * nz)
    assert np.sum(counts > 8) <= 1
    assert np.all(np.isfinite(pos))
    assert all(s.sdf.sample(p) < s.sdf.dx for p in pos)
    s2 = box_solver()
    pack_one_cell(s2, (8, 8, 8), N)
    s2.phase(oracle.PHASE_REDISTRIBUTE)
    assert np.array_equal(pos.view(np.uint64), s2.particles()[0].view(np.uint64))


def test_injection_stops_at_inject_until():  # solver.rs:1075-1099
    s = box_solver()
    n = s.needle
    s.set_needle(oracle.Needle(n.tip, n.axis, n.radius, n.flow_rate, 0.02))
    for _ in range(10):
        s.step(0.005)
    after = len(s)
    assert after > 0
    assert s.scalars()["time"] > 0.02
    for _ in range(10):
        s.step(0.005)
    assert len(s) == after


@pytest.fixture(scope="module")
def small_solver_sdf():  # solver.rs:1016-1043: Sdf::from_mesh(params.generate(), 2.5 mm, 6 mm)
    p = sc.SinusParams()
    tris = oracle.sinus_mesh(p)
    return p, oracle.sdf_from_mesh(tris, 0.0025, 0.006)


def small_solver(p, sdf):
    tip, axis = p.suggested_needle()
    s = oracle.Solver(sdf, 0.0025, oracle.Fluid(particles_per_cell=16), oracle.Needle(tip, axis, 0.0006, 5.0e-6))
    sx, sz = p.socket_xz
    yb = p.socket_bottom_y()
    s.set_outlet(((sx - 0.004, yb - 0.002, sz - 0.004), (sx + 0.004, yb + 0.002, sz + 0.004)))
    return s


def test_emits_fills_and_stays_out_of_walls(small_solver_sdf):  # solver.rs:1059-1118
    p, sdf = small_solver_sdf
    s = small_solver(p, sdf)
    for _ in range(12):
        s.step(0.005)
    pos, _ = s.particles()
    assert len(pos) > 0 and np.all(np.isfinite(pos))
    assert max(sdf.sample(q) for q in pos) < sdf.dx


def test_simulation_is_bit_reproducible(small_solver_sdf):  # solver.rs:1127-1164
    p, sdf = small_solver_sdf

    def run():
        s = small_solver(p, sdf)
        for _ in range(16):
            s.step(0.005)
        return s.particles()[0], s.pressure()

    pa, qa = run()
    pb, qb = run()
    assert pa.shape == pb.shape
    assert np.array_equal(pa.view(np.uint64), pb.view(np.uint64))
    assert np.array_equal(qa.view(np.uint64), qb.view(np.uint64))


# ---------------------------------------------------------------- pressure.rs
def classify_box(n):  # pressure.rs:755-770
    cells = np.full((n, n, n), oracle.FLUID, dtype=np.uint8)
    cells[0, :, :] = cells[-1, :, :] = cells[:, 0, :] = cells[:, -1, :] = cells[:, :, 0] = cells[:, :, -1] = oracle.SOLID
    return cells.reshape(-1)


def fill_divergent(n):  # pressure.rs:645-670
    u = np.zeros((n, n, n + 1))
    v = np.zeros((n, n + 1, n))
    w = np.zeros((n + 1, n, n))
    for k in range(n):
        for j in range(n):
            for i in range(n + 1):
                u[k, j, i] = (i - 6.0) * 0.05 + math.sin(j * 0.013)
    for k in range(n):
        for j in range(n + 1):
            for i in range(n):
                v[k, j, i] = (j - 6.0) * 0.05 + math.cos(k * 0.017)
    for k in range(n + 1):
        for j in range(n):
            for i in range(n):
                w[k, j, i] = (k - 6.0) * 0.03
    return u, v, w


def test_projection_is_idempotent():  # pressure.rs:619-642
    n = 12
    u, v, w = fill_divergent(n)
    cells = classify_box(n)
    u1, v1, w1, *_ = oracle.project(n, n, n, 0.01, u, v, w, cells, 1000.0, 1e-3, 400, 1e-12)
    u2, v2, w2, *_ = oracle.project(n, n, n, 0.01, u1, v1, w1, cells, 1000.0, 1e-3, 400, 1e-12)
    change = max(np.abs(u2 - u1).max(), np.abs(v2 - v1).max(), np.abs(w2 - w1).max())
    assert change < 1e-7


def test_removes_divergence():  # pressure.rs:675-723
    n = 12
    u = np.zeros((n, n, n + 1))
    v = np.zeros((n, n + 1, n))
    w = np.zeros((n + 1, n, n))
    u[:] = (np.arange(n + 1) - 6.0)[None, None, :] * 0.05
    v[:] = (np.arange(n + 1) - 6.0)[None, :, None] * 0.05
    u, v, w, p, iters, res = oracle.project(n, n, n, 0.01, u, v, w, classify_box(n), 1000.0, 1e-3, 400, 1e-9)
    u = u.reshape(n, n, n + 1)
    v = v.reshape(n, n + 1, n)
    w = w.reshape(n + 1, n, n)
    div = (u[1:-1, 1:-1, 2:-1] - u[1:-1, 1:-1, 1:-2]) + (v[1:-1, 2:-1, 1:-1] - v[1:-1, 1:-2, 1:-1]) + \
          (w[2:-1, 1:-1, 1:-1] - w[1:-2, 1:-1, 1:-1])
    assert np.abs(div).max() < 1e-5


def test_pressure_solve_is_bit_reproducible():  # pressure.rs:731-752
    n = 24
    u, v, w = fill_divergent(n)
    cells = classify_box(n)
    pa = oracle.project(n, n, n, 0.01, u, v, w, cells, 1000.0, 1e-3, 400, 1e-12)[3]
    oracle.set_threads(3)
    pb = oracle.project(n, n, n, 0.01, u, v, w, cells, 1000.0, 1e-3, 400, 1e-12)[3]
    oracle.set_threads(0)
    assert np.array_equal(pa.view(np.uint64), pb.view(np.uint64))


# ---------------------------------------------------------------- grid.rs
def test_constant_field_samples_exactly():  # grid.rs:215-224
    sdf = oracle.sdf_from_fn((0, 0, 0), 0.1, (9, 9, 9), lambda p: 3.0)
    assert abs(sdf.sample((0.41, 0.37, 0.55)) - 3.0) < 1e-9


# ---------------------------------------------------------------- metrics.rs
def test_membrane_stats_excludes_nonphysical_artifacts():  # metrics.rs:537-551
    mean, peak, art = oracle.membrane_stats([100.0, 200.0, 500.0, 900.0, 2_000_000.0], 1000.0)
    assert art == 1 and peak == 900.0
    assert abs(mean - (100.0 + 200.0 + 500.0 + 900.0) / 4.0) < 1e-9
    assert oracle.membrane_stats([10.0, 950.0], 1000.0) == (480.0, 950.0, 0)
    assert oracle.membrane_stats([5000.0], 1000.0) == (0.0, 0.0, 1)
    assert oracle.membrane_stats([], 1000.0) == (0.0, 0.0, 0)


def test_collector_records_and_summarises():  # metrics.rs:487-534
    cfg = sc.SceneConfig.from_toml_str("[sim]\nresolution_mm = 2.5\nduration_s = 0.04\nframes = 4\n[needle]\n"
                                       "auto = true\ndiameter_mm = 1.2\nflow_rate_ml_s = 5.0\n[fluid]\n"
                                       "particles_per_cell = 16\n")
    res = cfg.resolve()
    s = oracle_solver(res)
    m = oracle.Metrics(s, cavity_volume(res))
    assert m.wall_count > 0
    for f in range(res.frames):
        s.step(res.frame_dt)
        r = m.record(s, f)
        assert r["fill_fraction"] >= 0 and 0 <= r["wall_coverage"] <= 1
        assert r["peak_wall_pressure_pa"] <= r["max_pressure_pa"] + 1e-6
        assert r["wall_pressure_pa"] <= r["peak_wall_pressure_pa"] + 1e-6
    sm = m.summary()
    assert sm["frames"] == res.frames and sm["injected_ml"] > 0 and sm["peak_wall_coverage"] > 0
    assert sm["peak_membrane_pressure_pa"] <= sm["peak_pressure_pa"] + 1e-6
    assert sm["membrane_artifacts_total"] <= sm["frames"] * 2


# ---------------------------------------------------------------- sinus.rs / scene.rs
def test_generates_closed_cavity():  # sinus.rs:183-197
    vol, nt = oracle.sinus_mesh_volume(sc.SinusParams())
    assert 4.0 < vol * 1e6 < 35.0 and nt > 0


def test_needle_tip_is_inside_cavity():  # sinus.rs:200-209
    p = sc.SinusParams()
    tip, axis = p.suggested_needle()
    assert oracle.sinus_implicit(p, tip) < 0 and axis[1] > 0


def test_socket_is_below_body():  # sinus.rs:212-222
    p = sc.SinusParams()
    assert oracle.sinus_implicit(p, (p.socket_xz[0], p.socket_bottom_y() + 0.001, p.socket_xz[1])) < 0


def test_python_bounds_match_oracle():
    p = sc.SinusParams()
    mn, mx = oracle.sinus_bounds(p)
    pmn, pmx = p.bounds()
    assert np.array_equal(mn, np.array(pmn)) and np.array_equal(mx, np.array(pmx))
