"""GPU parity of the SDF builders, the cavity volume and the frame metrics,
plus run-to-run determinism (whole runs against the oracle: test_gpu_whole_run.py)."""
import numpy as np
import pytest

import oracle
from sdr_b200 import scene as sc
from sdr_b200.cavity import perturbed_ellipsoid
from tests.gpu_common import SMOKE_TOML, make_pair, record, rel_err
from tests.helpers import cavity_volume, oracle_solver
from tests.test_oracle_kats import box_tris

pytestmark = pytest.mark.gpu


def test_winding_sdf_box_known_answers():  # sdf.rs:298-335 on the device
    from sdr_b200.solver import sdf_from_mesh
    sdf = sdf_from_mesh(box_tris(), 0.5, 2.5)
    o = np.asarray(sdf.origin)
    assert np.allclose(o, -3.5)
    nz, ny, nx = sdf.data.shape
    ic = int(round((0.0 - o[0]) / 0.5))
    io = int(round((3.0 - o[0]) / 0.5))
    assert sdf.data[ic, ic, ic] == -1.0
    assert sdf.data[ic, ic, io] == 2.0


def test_winding_sdf_matches_oracle():
    """Sign bit-exact; distance bit-exact (same f64 closest-point arithmetic)."""
    from sdr_b200.solver import sdf_from_mesh
    cav = perturbed_ellipsoid(7, subdiv=3)
    g = sdf_from_mesh(cav.tris, 1.0e-3, 3.0e-3)
    o = oracle.sdf_from_mesh(cav.tris, 1.0e-3, 3.0e-3)
    assert g.data.shape == o.data.shape
    assert np.allclose(np.asarray(g.origin), o.origin, rtol=0, atol=0)
    sign_mismatch = int(np.sum(np.signbit(g.data) != np.signbit(o.data)))
    dist_mismatch = int(np.sum(np.abs(g.data) != np.abs(o.data)))
    record("sdf_mesh", {"nodes": int(g.data.size), "tris": int(len(cav.tris)), "sign_mismatch": sign_mismatch,
                        "dist_mismatch": dist_mismatch, "max_abs_diff": float(np.abs(g.data - o.data).max())})
    assert sign_mismatch == 0
    assert dist_mismatch == 0


def test_sinus_sdf_matches_oracle():
    """Parametric implicit on the device vs glibc: within a few ulps (sin/cos)."""
    from sdr_b200.solver import sdf_from_sinus
    res = sc.SceneConfig.from_toml_str("").resolve()
    g = sdf_from_sinus(res.sinus, res.sdf_origin, res.sdf_dx, res.sdf_dims)
    o = oracle.sdf_from_sinus(res.sinus, res.sdf_origin, res.sdf_dx, res.sdf_dims)
    d = float(np.abs(g.data - o.data).max())
    record("sdf_sinus", {"nodes": int(g.data.size), "max_abs_diff": d})
    assert d < 1e-16
    assert np.array_equal(g.data < 0, o.data < 0)


def test_surface_nets_volume_matches_oracle():
    from sdr_b200.solver import Sdf, surface_nets_volume
    res = sc.SceneConfig.from_toml_str("").resolve()
    o = oracle.sdf_from_sinus(res.sinus, res.sdf_origin, res.sdf_dx, res.sdf_dims)
    v = surface_nets_volume(Sdf(tuple(o.origin), o.dx, o.data))
    vo, _ = oracle.sinus_mesh_volume(res.sinus)
    assert v == vo


def test_metrics_match_oracle():
    """MetricsCollector::record on the device vs the oracle from the same state."""
    from sdr_b200.solver import MetricsCollector
    gpu, orc, res = make_pair(warm_frames=3)
    dt = orc.cfl_dt()
    vol = cavity_volume(res)
    mg = MetricsCollector(gpu, vol)
    mo = oracle.Metrics(orc, vol)
    assert mg.wall_count == mo.wall_count
    gpu.substep(dt)
    orc.substep(dt)
    fg = mg.record(gpu, 0)
    fo = mo.record(orc, 0)
    record("metrics", {"gpu": fg, "orc": fo})
    for k in ("particles", "fill_fraction", "fluid_volume_ml", "drained_volume_ml", "pcg_iters"):
        assert fg[k] == fo[k], k
    assert abs(fg["wall_coverage"] - fo["wall_coverage"]) < 1e-3
    for k in ("mean_pressure_pa", "max_pressure_pa", "wall_pressure_pa", "peak_wall_pressure_pa"):
        assert abs(fg[k] - fo[k]) <= 1e-4 * max(abs(fo[k]), 1.0), (k, fg[k], fo[k])
    assert abs(fg["kinetic_energy"] - fo["kinetic_energy"]) <= 1e-5 * fo["kinetic_energy"]
    assert abs(fg["max_speed_m_s"] - fo["max_speed_m_s"]) <= 1e-5 * fo["max_speed_m_s"]


def _run(frames=2):
    from sdr_b200.solver import build_scene
    b = build_scene(sc.SceneConfig.from_toml_str(SMOKE_TOML))
    for _ in range(frames):
        b.solver.step(b.frame_dt)
    p, v = b.solver.particles()
    return p, v, b.solver.pressure()


def test_gpu_is_byte_identical_run_to_run():  # solver.rs:1127-1164 on the device
    a = _run()
    b = _run()
    for x, y in zip(a, b):
        assert x.shape == y.shape
        assert np.array_equal(x.view(np.uint64), y.view(np.uint64))
