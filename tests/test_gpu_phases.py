"""Per-phase parity of the CUDA substep against the CPU oracle (shadow stepping).

Every phase test runs on each state of tests/gpu_states.py: the CI smoke
scene, the 0.8 mm parametric jet, the 0.5 mm perturbed-ellipsoid cavity while
the jet fires and after it has settled, and the 0.2 mm pre-seeded pool of
9.5 M particles. Before each phase both solvers hold identical state (the
device's f32 values, widened to f64 for the oracle); after it the outputs are
compared:
  * integer work (labels, cell keys, the counting-sort permutation, the
    bounds/compaction map, redistribution moves) and the CFL step - bit-exact;
  * the pressure solve - bit-exact pressure and iteration count with the
    reference dot order, because the device repeats the reference's f64
    arithmetic;
  * f32 transfers (P2G, extrapolation, G2P, advection) - the largest error
    over every face or particle, within the tolerances stated below, against
    the oracle's f64 arithmetic.
"""
import numpy as np
import pytest

import oracle
from sdr_b200 import _lib
from tests.gpu_common import f32, make_pair, record, rel_err
from tests.gpu_states import STATES, gpu_to_oracle, make_state, sync_faces

pytestmark = pytest.mark.gpu

FACE_TOL = 2e-6      # f32 face values vs f64 (relative to the field's max)
P2G_TOL = 1e-6       # P2G faces, absolute error relative to the particles' max speed: f32
                     # weights of faces whose weighted velocities cancel carry ~1e-7 of
                     # the particle speed, not of the (small) face value
VEL_TOL = 2e-5       # particle velocities (relative to max speed)
POS_TOL = 1e-7       # particle positions, metres (f32 spacing at 2 cm is ~1.9e-9 m)


@pytest.fixture(scope="module", params=STATES)
def pair(request):
    gpu, orc, res = make_state(request.param)
    assert len(gpu) > 100
    yield gpu, orc, res, request.param
    gpu.close()


def test_cfl_step_bit_exact(pair):
    """cfl_dt (solver.rs:262-281) from MacGrid::max_speed (grid.rs:202-206):
    the device reduces the face maxima in the last extrapolation sweep and
    combines them on the host in f64. On the same (f32) faces that is the
    oracle's dt and grid speed bit for bit; against the oracle's own f64
    extrapolation the grid speed differs by the f32 rounding of the faces."""
    gpu, orc, res, name = pair
    sync_faces(gpu, orc)
    gpu.run_phase(_lib.PHASE_EXTRAPOLATE)
    orc.phase(oracle.PHASE_EXTRAPOLATE)
    own = orc.grid_max_speed()
    sync_faces(gpu, orc, (0, 1, 2))
    dt_g, gs_g = gpu.cfl()
    dt_o, gs_o = orc.cfl_dt(), orc.grid_max_speed()
    record(f"cfl[{name}]", {"dt_gpu": dt_g, "dt_orc": dt_o, "speed_gpu": gs_g, "speed_orc": gs_o,
                             "speed_orc_f64_faces": own})
    assert gs_g == gs_o
    assert dt_g == dt_o
    assert abs(gs_g - own) <= 1e-6 * max(own, 1e-30)


def test_classify_labels_bit_exact(pair):
    gpu, orc, res, name = pair
    gpu.run_phase(_lib.PHASE_CLASSIFY)
    orc.phase(oracle.PHASE_CLASSIFY)
    g, o = gpu.cells(), orc.cells()
    record(f"classify[{name}]", {"cells": int(g.size), "fluid": int((o == 1).sum()), "mismatch": int((g != o).sum())})
    assert np.array_equal(g, o)
    assert np.array_equal(gpu.cavity_mask(), orc.cavity_mask())


def test_p2g_sort_is_stable_counting_sort(pair):
    gpu, orc, res, name = pair
    gpu.run_phase(_lib.PHASE_P2G)
    keys, perm = gpu.sort()
    # CPU stable counting sort of the same keys
    ref = np.argsort(keys, kind="stable").astype(np.uint32)
    record(f"sort[{name}]", {"n": int(keys.size), "perm_mismatch": int((perm != ref).sum())})
    assert np.array_equal(perm, ref)
    # the keys are the cell of each particle's f64 grid coordinate (p - origin) / dx
    # of its stored f32 position, clamped to the grid (k_classify_keys)
    pos, _ = gpu.particles()
    (nx, ny, nz) = gpu.grid_dims
    st = gpu.stats()
    o = np.array([st.origin.x, st.origin.y, st.origin.z], dtype=np.float64)
    l = (pos - o) / st.dx
    ijk = np.where(l > 0, np.floor(l), 0).astype(np.int64)
    ijk = np.minimum(ijk, np.array([nx - 1, ny - 1, nz - 1]))
    k2 = (ijk[:, 2] * ny + ijk[:, 1]) * nx + ijk[:, 0]
    assert np.array_equal(keys.astype(np.int64), k2)


def test_p2g_faces(pair):
    gpu, orc, res, name = pair
    gpu.run_phase(_lib.PHASE_P2G)
    orc.phase(oracle.PHASE_P2G)
    orc.phase(oracle.PHASE_SAVE_GRID)
    _, vel = gpu.particles()
    vscale = float(np.max(np.abs(vel)))
    errs = {w: float(np.max(np.abs(gpu.face(w) - orc.face(w)))) / vscale for w in range(6)}
    record(f"p2g[{name}]", {"err_over_vmax": errs, "vmax": vscale})
    for w in range(6):
        assert errs[w] < P2G_TOL, errs


def test_add_forces(pair):
    gpu, orc, res, name = pair
    dt = 1e-4
    sync_faces(gpu, orc)
    gpu.run_phase(_lib.PHASE_ADD_FORCES, dt)
    orc.phase(oracle.PHASE_ADD_FORCES, dt)
    for w in range(3):
        assert rel_err(gpu.face(w), orc.face(w)) < FACE_TOL


def test_project_bit_exact_pressure(pair):
    """With the reference dot order the solve is bit-exact: same iterations, same pressure bits."""
    gpu, orc, res, name = pair
    dt = 1e-4
    gpu.set_dot_order(True)
    gpu.run_phase(_lib.PHASE_CLASSIFY)
    orc.phase(oracle.PHASE_CLASSIFY)
    sync_faces(gpu, orc)
    gpu.run_phase(_lib.PHASE_PROJECT, dt)
    orc.phase(oracle.PHASE_PROJECT, dt)
    pg, po = gpu.pressure(), orc.pressure()
    it_g, it_o = gpu.last_pcg_iters, orc.scalars()["last_pcg_iters"]
    diff = int(np.sum(pg.view(np.uint64) != po.view(np.uint64)))
    errs = {w: rel_err(gpu.face(w), orc.face(w)) for w in range(3)}
    record(f"project[{name}]", {"iters_gpu": it_g, "iters_orc": it_o, "pressure_bit_mismatch": diff,
                       "pressure_rel_err": rel_err(pg, po), "max_p": float(po.max()), "face_rel_err": errs})
    gpu.set_dot_order(False)
    assert it_g == it_o
    assert diff == 0
    for w in range(3):
        assert errs[w] < FACE_TOL


WIDE_TOML = """
[sim]
resolution_mm = 0.6
duration_s = 0.5
frames = 10
[needle]
auto = true
diameter_mm = 0.8
flow_rate_ml_s = 5.0
"""


def _wide_pair():
    """The parametric cavity filled with fluid at 0.6 mm (one particle per cell
    centre) and random faces: a solve whose wavefront levels are wider than the
    one-block kernel's shared-memory window."""
    gpu, orc, res = make_pair(WIDE_TOML)
    (nx, ny, nz), origin, dx = orc.grid
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    pos = np.stack([origin[0] + (i + 0.5) * dx, origin[1] + (j + 0.5) * dx, origin[2] + (k + 0.5) * dx],
                   axis=-1).reshape(-1, 3)
    pos = f32(pos)
    vel = np.zeros_like(pos)
    gpu.set_particles(pos, vel)
    orc.set_particles(pos, vel)
    rng = np.random.default_rng(5)
    for w in range(3):
        f = f32(0.05 * rng.standard_normal(orc.face(w).shape))
        gpu.set_face(w, f)
        orc.set_face(w, f)
    gpu.run_phase(_lib.PHASE_CLASSIFY)
    orc.phase(oracle.PHASE_CLASSIFY)
    fluid = orc.cells().reshape(nz, ny, nx) == 1
    widths = np.bincount((i + j + k)[fluid])
    sync_faces(gpu, orc)
    return gpu, orc, fluid, widths


@pytest.mark.parametrize("kernel", [_lib.PCG_ONE_BLOCK, _lib.PCG_CLUSTER, _lib.PCG_TILES],
                         ids=["one_block", "cluster", "tiles"])
def test_project_wide_levels_bit_exact(kernel):
    """Wide wavefront levels: the one-block kernel takes its global-memory path
    for them (and the window path around them); the cluster kernel spreads
    every level over its CTAs; the tiled kernel walks 16 x 16-line tiles over
    the whole GPU, handing boundary values between tiles. With the reference
    dot order all three give the reference's pressure and iteration count bit
    for bit."""
    gpu, orc, fluid, widths = _wide_pair()
    gpu.set_dot_order(True)
    gpu.set_pcg_kernel(kernel)
    gpu.set_profiling(True)
    gpu.run_phase(_lib.PHASE_PROJECT, 1e-4)
    orc.phase(oracle.PHASE_PROJECT, 1e-4)
    prof = gpu.profile()
    pg, po = gpu.pressure(), orc.pressure()
    it_g, it_o = gpu.last_pcg_iters, orc.scalars()["last_pcg_iters"]
    diff = int(np.sum(pg.view(np.uint64) != po.view(np.uint64)))
    name = {_lib.PCG_ONE_BLOCK: "project_wide", _lib.PCG_CLUSTER: "project_wide_cluster",
            _lib.PCG_TILES: "project_wide_tiles"}[kernel]
    record(name, {"fluid_cells": int(fluid.sum()), "max_level_width": int(widths.max()),
                  "levels_over_736": int((widths > 736).sum()), "iters_gpu": it_g, "iters_orc": it_o,
                  "pressure_bit_mismatch": diff, "pcg_ms": prof["pcg_ms"]})
    assert prof["pcg_cluster_launches"] == (1 if kernel == _lib.PCG_CLUSTER else 0)
    assert prof["pcg_tile_launches"] == (1 if kernel == _lib.PCG_TILES else 0)
    assert widths.max() > 768
    assert it_g == it_o
    assert diff == 0


def test_project_tree_dots_same_bits_for_every_kernel():
    """The default tree-order dots do not depend on where the solve runs:
    sweeps on one SM with the rest on 1, 2 or 4 CTAs or the device's largest
    cluster, everything on the cluster kernel, or the tiled solve over the
    whole GPU, give the same pressure bits and iteration count."""
    runs = {}
    for name, kernel, ctas in [("one_cta", _lib.PCG_ONE_BLOCK, 1), ("two_ctas", _lib.PCG_ONE_BLOCK, 2),
                               ("four_ctas", _lib.PCG_ONE_BLOCK, 4), ("auto", _lib.PCG_ONE_BLOCK, 0),
                               ("cluster", _lib.PCG_CLUSTER, 0), ("tiles", _lib.PCG_TILES, 0)]:
        gpu, orc, fluid, widths = _wide_pair()
        gpu.set_pcg_kernel(kernel)
        gpu.set_pcg_ctas(ctas)
        gpu.run_phase(_lib.PHASE_PROJECT, 1e-4)
        runs[name] = (gpu.pressure(), gpu.last_pcg_iters)
    ref_p, ref_it = runs["one_cta"]
    record("project_tree_kernels", {k: {"iters": it, "bit_mismatch": int(np.sum(p.view(np.uint64) != ref_p.view(np.uint64)))}
                                    for k, (p, it) in runs.items()})
    for name, (p, it) in runs.items():
        assert it == ref_it, name
        assert np.array_equal(p.view(np.uint64), ref_p.view(np.uint64)), name


def test_project_cluster_tree_dots():
    """The cluster kernel with its default tree dots (per-CTA trees added in
    CTA order): pressure within the tree-order tolerance of the reference."""
    gpu, orc, fluid, widths = _wide_pair()
    gpu.set_pcg_kernel(_lib.PCG_CLUSTER)
    gpu.run_phase(_lib.PHASE_PROJECT, 1e-4)
    orc.phase(oracle.PHASE_PROJECT, 1e-4)
    pg, po = gpu.pressure(), orc.pressure()
    it_g, it_o = gpu.last_pcg_iters, orc.scalars()["last_pcg_iters"]
    e = rel_err(pg, po)
    record("project_cluster_tree", {"iters_gpu": it_g, "iters_orc": it_o, "pressure_rel_err": e})
    assert abs(it_g - it_o) <= 1
    assert e < PRESSURE_TOL


PRESSURE_TOL = 1e-8  # block-tree dots: pressure relative to its max, f64


def test_project_tree_dots(pair):
    """The default block-tree dot order: pressure within 1e-8 relative, iterations within one."""
    gpu, orc, res, name = pair
    dt = 1e-4
    gpu.run_phase(_lib.PHASE_CLASSIFY)
    orc.phase(oracle.PHASE_CLASSIFY)
    sync_faces(gpu, orc)
    gpu.run_phase(_lib.PHASE_PROJECT, dt)
    orc.phase(oracle.PHASE_PROJECT, dt)
    pg, po = gpu.pressure(), orc.pressure()
    it_g, it_o = gpu.last_pcg_iters, orc.scalars()["last_pcg_iters"]
    e = rel_err(pg, po)
    record(f"project_tree[{name}]", {"iters_gpu": it_g, "iters_orc": it_o, "pressure_rel_err": e})
    assert abs(it_g - it_o) <= 1
    assert e < PRESSURE_TOL


def test_extrapolate(pair):
    gpu, orc, res, name = pair
    sync_faces(gpu, orc)
    gpu.run_phase(_lib.PHASE_EXTRAPOLATE)
    orc.phase(oracle.PHASE_EXTRAPOLATE)
    errs = {w: rel_err(gpu.face(w), orc.face(w)) for w in range(3)}
    record(f"extrapolate[{name}]", {"rel_err": errs})
    for w in range(3):
        assert errs[w] < FACE_TOL


def test_g2p(pair):
    gpu, orc, res, name = pair
    sync_faces(gpu, orc)
    pos, vel = gpu.particles()
    orc.set_particles(pos, vel)
    gpu.run_phase(_lib.PHASE_G2P)
    orc.phase(oracle.PHASE_G2P)
    _, vg = gpu.particles()
    _, vo = orc.particles()
    e = rel_err(vg, vo)
    record(f"g2p[{name}]", {"n": int(len(vg)), "vel_rel_err": e})
    assert e < VEL_TOL


def test_advect(pair):
    gpu, orc, res, name = pair
    dt = 1e-4
    sync_faces(gpu, orc)
    pos, vel = gpu.particles()
    orc.set_particles(pos, vel)
    gpu.run_phase(_lib.PHASE_ADVECT, dt)
    orc.phase(oracle.PHASE_ADVECT, dt)
    pg, _ = gpu.particles()
    po, _ = orc.particles()
    d = np.max(np.abs(pg - po), axis=1)
    record(f"advect[{name}]", {"n": int(len(d)), "max_abs": float(d.max()), "p99": float(np.quantile(d, 0.99)),
                               "n_over_tol": int((d > POS_TOL).sum())})
    assert d.max() < POS_TOL


def test_bounds_compaction_exact(pair):
    gpu, orc, res, name = pair
    pos, vel = gpu.particles()
    orc.set_particles(pos, vel)
    d0g, d0o = gpu.drained, orc.scalars()["drained"]
    gpu.run_phase(_lib.PHASE_BOUNDS)
    orc.phase(oracle.PHASE_BOUNDS)
    pg, vg = gpu.particles()
    po, vo = orc.particles()
    record(f"bounds[{name}]", {"n_gpu": int(len(pg)), "n_orc": int(len(po)), "drained_gpu": gpu.drained - d0g,
                      "drained_orc": orc.scalars()["drained"] - d0o})
    assert len(pg) == len(po)
    assert np.array_equal(pg, po)  # same survivors, same order, same (f32) values
    assert np.array_equal(vg, vo)


def test_redistribute_moves_exact(pair):
    gpu, orc, res, name = pair
    sync_faces(gpu, orc)
    pos, vel = gpu.particles()
    orc.set_particles(pos, vel)
    gpu.run_phase(_lib.PHASE_REDISTRIBUTE)
    orc.phase(oracle.PHASE_REDISTRIBUTE)
    pg, vg = gpu.particles()
    po, vo = orc.particles()
    moved_g = np.any(pg != pos, axis=1)
    moved_o = np.any(po != pos, axis=1)
    d = np.max(np.abs(pg - po), axis=1)
    record(f"redistribute[{name}]", {"moved_gpu": int(moved_g.sum()), "moved_orc": int(moved_o.sum()),
                            "max_abs_pos": float(d.max()) if len(d) else 0.0,
                            "vel_rel_err": rel_err(vg, vo)})
    assert np.array_equal(moved_g, moved_o)
    assert d.max() < POS_TOL


def test_redistribute_long_candidate_list_exact():
    """More over-cap particles than the replay keeps in shared memory (8192):
    24 particles in every cavity cell of even i+j+k and none in the others (a
    checkerboard, so every over-cap cell has room next to it and no candidate
    is left out), in shuffled index order. The list is put in index order
    through the bitmap and the moves are decided in parallel rounds on a
    cluster (k_redist_par): the same moves as the reference's sequential loop."""
    gpu, orc, res = make_pair()
    nx, ny, nz = gpu.grid_dims
    dx = gpu.dx
    st = gpu.stats()
    org = np.array([st.origin.x, st.origin.y, st.origin.z])
    cav = np.flatnonzero(gpu.cavity_mask().reshape(-1))
    ijk = np.stack([cav % nx, (cav // nx) % ny, cav // (nx * ny)], axis=1)
    ijk = ijk[ijk.sum(axis=1) % 2 == 0]
    assert len(ijk) * 24 > 8192
    rng = np.random.default_rng(7)
    pos = (org + (ijk.repeat(24, axis=0) + 0.5 + rng.uniform(-0.3, 0.3, (len(ijk) * 24, 3))) * dx)
    pos = f32(pos[rng.permutation(len(pos))])
    vel = np.zeros_like(pos)
    gpu.set_particles(pos, vel)
    orc.set_particles(pos, vel)
    sync_faces(gpu, orc)
    gpu.set_profiling(True)
    gpu.run_phase(_lib.PHASE_REDISTRIBUTE)
    orc.phase(oracle.PHASE_REDISTRIBUTE)
    prof = gpu.profile()
    pg, vg = gpu.particles()
    po, vo = orc.particles()
    moved_g = np.any(pg != pos, axis=1)
    moved_o = np.any(po != pos, axis=1)
    d = np.max(np.abs(pg - po), axis=1)
    record("redistribute_long", {"particles": int(len(pos)), "candidates": prof["redist_candidates"],
                                 "sweeps": prof["redist_sweeps"], "long_sweeps": prof["redist_long_sweeps"],
                                 "moved_gpu": int(moved_g.sum()), "moved_orc": int(moved_o.sum()),
                                 "max_abs_pos": float(d.max())})
    assert prof["redist_long_sweeps"] >= 1
    assert moved_o.sum() > 1000
    assert np.array_equal(moved_g, moved_o)
    assert d.max() < POS_TOL


def test_redistribute_crowded_cells_exact():
    """A jet's pile-up: 500 particles in each of three adjacent cavity cells
    deep inside the cavity (a short list, replayed in shared memory). Each
    round can move one candidate per crowded cell, so the first round decides
    fewer than 32 and thread 0 decides the pending rest in index order: the
    same moves as the reference's sequential loop (solver.rs:476-555)."""
    gpu, orc, res = make_pair()
    nx, ny, nz = gpu.grid_dims
    dx = gpu.dx
    st = gpu.stats()
    org = np.array([st.origin.x, st.origin.y, st.origin.z])
    cav = gpu.cavity_mask().reshape(nz, ny, nx).astype(bool)
    inner = cav.copy()
    for ax in range(3):
        for sh in (-1, 1):
            inner &= np.roll(cav, sh, axis=ax)
    inner[:, :, :2] = inner[:, :, -2:] = False
    row = inner[:, :, 1:-1] & inner[:, :, :-2] & inner[:, :, 2:]
    kk, jj, ii = np.argwhere(row)[len(np.argwhere(row)) // 2]
    cells = np.array([[ii, jj, kk], [ii + 1, jj, kk], [ii + 2, jj, kk]])
    rng = np.random.default_rng(3)
    pos = org + (cells.repeat(500, axis=0) + 0.5 + rng.uniform(-0.3, 0.3, (1500, 3))) * dx
    pos = f32(pos[rng.permutation(len(pos))])
    vel = np.zeros_like(pos)
    gpu.set_particles(pos, vel)
    orc.set_particles(pos, vel)
    sync_faces(gpu, orc)
    gpu.set_profiling(True)
    gpu.run_phase(_lib.PHASE_REDISTRIBUTE)
    orc.phase(oracle.PHASE_REDISTRIBUTE)
    prof = gpu.profile()
    pg, vg = gpu.particles()
    po, vo = orc.particles()
    moved_g = np.any(pg != pos, axis=1)
    moved_o = np.any(po != pos, axis=1)
    d = np.max(np.abs(pg - po), axis=1)
    record("redistribute_crowded", {"particles": int(len(pos)), "candidates": prof["redist_candidates"],
                                    "sweeps": prof["redist_sweeps"], "long_sweeps": prof["redist_long_sweeps"],
                                    "moved_gpu": int(moved_g.sum()), "moved_orc": int(moved_o.sum()),
                                    "max_abs_pos": float(d.max())})
    assert prof["redist_long_sweeps"] == 0
    assert moved_o.sum() > 20
    assert np.array_equal(moved_g, moved_o)
    assert d.max() < POS_TOL


def test_redistribute_table_overflow_exact():
    """A short list (at most 8192 candidates) whose cells do not fit the
    replay's 4096-slot shared table: 9 to 11 particles in each of 700 cavity
    cells three apart on every axis (4900 distinct cells with their
    neighbours), at 0.6 mm. The replay hands the list to k_redist_par, which
    decides it in rounds: the same moves as the reference's sequential loop."""
    import re

    from tests.gpu_common import SMOKE_TOML
    gpu, orc, res = make_pair(re.sub(r"resolution_mm = [0-9.]+", "resolution_mm = 0.6", SMOKE_TOML))
    nx, ny, nz = gpu.grid_dims
    dx = gpu.dx
    st = gpu.stats()
    org = np.array([st.origin.x, st.origin.y, st.origin.z])
    cav = gpu.cavity_mask().reshape(nz, ny, nx).astype(bool)
    inner = cav.copy()
    for ax in range(3):
        for sh in (-1, 1):
            inner &= np.roll(cav, sh, axis=ax)
    lat = np.zeros_like(inner)
    lat[1::3, 1::3, 1::3] = True
    kji = np.argwhere(inner & lat)
    assert len(kji) >= 700
    rng = np.random.default_rng(5)
    kji = kji[np.sort(rng.choice(len(kji), 700, replace=False))]
    per = rng.integers(9, 12, size=700)
    ijk = kji[:, ::-1].repeat(per, axis=0)
    pos = org + (ijk + 0.5 + rng.uniform(-0.3, 0.3, (len(ijk), 3))) * dx
    pos = f32(pos[rng.permutation(len(pos))])
    vel = np.zeros_like(pos)
    gpu.set_particles(pos, vel)
    orc.set_particles(pos, vel)
    sync_faces(gpu, orc)
    gpu.set_profiling(True)
    gpu.run_phase(_lib.PHASE_REDISTRIBUTE)
    orc.phase(oracle.PHASE_REDISTRIBUTE)
    prof = gpu.profile()
    pg, vg = gpu.particles()
    po, vo = orc.particles()
    moved_g = np.any(pg != pos, axis=1)
    moved_o = np.any(po != pos, axis=1)
    d = np.max(np.abs(pg - po), axis=1)
    record("redistribute_table_overflow", {"particles": int(len(pos)), "candidates": prof["redist_candidates"],
                                           "sweeps": prof["redist_sweeps"],
                                           "long_sweeps": prof["redist_long_sweeps"],
                                           "moved_gpu": int(moved_g.sum()), "moved_orc": int(moved_o.sum()),
                                           "max_abs_pos": float(d.max())})
    assert len(pos) <= 8192
    assert prof["redist_long_sweeps"] >= 1
    assert moved_o.sum() >= 700
    assert np.array_equal(moved_g, moved_o)
    assert d.max() < POS_TOL


SUB_POS_TOL = 1e-7      # one whole substep: particle positions, metres
SUB_VEL_TOL = 2e-5      # velocities, relative to the largest speed
SUB_PRESSURE_TOL = 1e-6  # pressure, relative to its largest value: the f32 faces of P2G move the RHS
# A particle that ends a substep within f32 rounding (~1e-9 m) of a cell face
# can be counted in the neighbouring cell on one side only; the redistribution
# sweep's decisions read those counts, so a handful of moves can then differ
# (each a jump of about a cell). At most this fraction of the particles may do
# so, each within two cells; every other particle holds the bounds above.
SUB_BRANCH_FRACTION = 1e-5
# PCG stops at the first iteration whose residual max-norm is below the
# absolute tolerance (pressure.rs:377-380). Over a whole substep the device's
# right-hand side comes from its f32 P2G faces and the oracle's from f64 faces
# (~1e-7 relative apart), which can move that iteration by one where the
# residual crosses the tolerance near the end (the 0.2 mm pool: 216 against
# 217, pressure still within 1.2e-8). From identical faces the project phase
# has equal iterations and identical pressure bits (test_project_*).
SUB_ITERS_SLACK = 1


def test_full_substep_shadow(pair):
    """One full substep from identical state, both in the reference dot order:
    particle count, labels and drained count exactly, PCG iterations within
    one; the pressure of every cell, and every particle's position and
    velocity but for the redistribution branch flips described above, within
    the stated bounds."""
    gpu, orc, res, name = pair
    gpu_to_oracle(gpu, orc)
    sync_faces(gpu, orc)
    dt = orc.cfl_dt()
    gpu.set_dot_order(True)
    gpu.substep(dt)
    gpu.set_dot_order(False)
    orc.substep(dt)
    pg, vg = gpu.particles()
    po, vo = orc.particles()
    pr_g, pr_o = gpu.pressure(), orc.pressure()
    rec = {"n_gpu": int(len(pg)), "n_orc": int(len(po)), "iters_gpu": gpu.last_pcg_iters,
           "iters_orc": orc.scalars()["last_pcg_iters"], "dt": dt, "drained_gpu": gpu.drained,
           "drained_orc": orc.scalars()["drained"]}
    if len(pg) == len(po):
        d = np.max(np.abs(pg - po), axis=1)
        vscale = max(float(np.max(np.abs(vo))), 1e-30)
        dv = np.max(np.abs(vg - vo), axis=1) / vscale
        dp = np.abs(pr_g - pr_o) / max(float(np.max(np.abs(pr_o))), 1e-30)
        flips = (d > SUB_POS_TOL) | (dv > SUB_VEL_TOL)
        rec.update(pos_max=float(d.max()), pos_p99=float(np.quantile(d, 0.99)),
                   pos_max_others=float(d[~flips].max()) if (~flips).any() else 0.0,
                   vel_rel_max=float(dv.max()), vel_rel_p99=float(np.quantile(dv, 0.99)),
                   vel_rel_max_others=float(dv[~flips].max()) if (~flips).any() else 0.0,
                   branch_flips=int(flips.sum()), flip_jump_max=float(d[flips].max()) if flips.any() else 0.0,
                   pressure_rel_max=float(dp.max()), pressure_rel_p99=float(np.quantile(dp, 0.99)),
                   vmax=vscale, pmax=float(np.max(np.abs(pr_o))))
    record(f"full_substep[{name}]", rec)
    assert len(pg) == len(po)
    assert gpu.drained == orc.scalars()["drained"]
    assert abs(rec["iters_gpu"] - rec["iters_orc"]) <= SUB_ITERS_SLACK
    assert np.array_equal(gpu.cells(), orc.cells())
    assert rec["pressure_rel_max"] < SUB_PRESSURE_TOL
    assert rec["branch_flips"] <= SUB_BRANCH_FRACTION * len(pg)
    assert rec["flip_jump_max"] <= 2.0 * res.sim_dx
    assert rec["pos_max_others"] < SUB_POS_TOL
    assert rec["vel_rel_max_others"] < SUB_VEL_TOL
