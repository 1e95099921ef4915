"""Host logic of the batch and serving layer, on the CPU.

No GPU here: a scene that reaches the device fails at solver creation with
a clear error, which is enough to exercise validation, the footprint
estimate, admission by budget and failure reporting."""
import ctypes as C

import numpy as np
import pytest

from sdr_b200 import _lib, scene as sc
from sdr_b200.serving import SceneSpec, Server, footprint, run_batch
from sdr_b200.solver import Sdf


def _spec(flow_ml_s=4.0, frames=2, n=24, dx=1e-3):
    # a sphere SDF of radius 8 mm on an n^3 node grid
    g = (np.arange(n) - (n - 1) / 2) * dx
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    data = np.sqrt(x * x + y * y + z * z) - 8e-3
    sdf = Sdf((float(g[0]),) * 3, dx, data)
    fluid = sc.FluidParams()
    needle = sc.Needle(tip=(0.0, -6e-3, 0.0), axis=(0.0, 1.0, 0.0), radius=4e-4,
                       flow_rate=flow_ml_s * sc.ML_PER_S, inject_until=0.25)
    return SceneSpec(sdf=sdf, sim_dx=dx, fluid=fluid, needle=needle, solve=sc.SolveParams(50, 1e-6),
                     cavity_volume=4.0 / 3.0 * np.pi * 8e-3 ** 3, frame_dt=0.01, frames=frames)


def test_footprint_counts_grid_and_dose():
    base = footprint(_spec())
    assert base > 16 << 20
    assert footprint(_spec(flow_ml_s=8.0)) > base          # more particles
    assert footprint(_spec(frames=10)) > base              # more of the dose injected
    assert footprint(_spec(n=40)) > base                   # more cells


def test_invalid_scene_is_rejected():
    s = _spec()
    s.frame_dt = 0.0
    with pytest.raises(_lib.SdrError):
        footprint(s)
    with pytest.raises(_lib.SdrError):
        run_batch([s])


def test_batch_reports_per_scene_errors_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("this test needs a machine without a GPU")
    res = run_batch([_spec(), _spec(flow_ml_s=6.0)], concurrency=2)
    assert len(res) == 2
    for r in res:
        assert r.status != _lib.SDR_OK and r.summary is None and r.error


def test_server_admission_and_failures_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("this test needs a machine without a GPU")
    big = footprint(_spec(n=40))
    with Server(budget_bytes=big - 1, max_active=2) as srv:
        t_big = srv.submit(_spec(n=40))        # can never fit: fails at once
        r = srv.poll(t_big)
        assert r.status == _lib.REQ_FAILED and "budget" in r.error
        tickets = [srv.submit(_spec(flow_ml_s=f)) for f in (2.0, 3.0, 4.0)]
        res = srv.wait(tickets, timeout=60)
        assert all(x.status == _lib.REQ_FAILED and x.error for x in res)  # no device here
        st = srv.stats()
        assert st["submitted"] == 4 and st["failed"] == 4 and st["completed"] == 0
        assert st["peak_active"] <= 2 and st["active"] == 0 and st["bytes_in_use"] == 0
        with pytest.raises(_lib.SdrError):
            srv.poll(12345)
