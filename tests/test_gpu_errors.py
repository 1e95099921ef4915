"""Device error paths, exercised without any GPU fault.

* A bounded wait that runs out: the test hook makes k_sdf_mesh skip the bulk
  copy of its first triangle tile, so the staging wait gives up after its
  limit (about a second); the kernel reports through its error word and the
  call returns SDR_ERR_DEVICE_TIMEOUT. The next call on the same context
  succeeds and matches the oracle.
* A work list that overflows: a redistribution candidate list smaller than a
  sweep's candidates makes the substep return SDR_ERR_CAPACITY; the solver
  stays usable, and with the default list the same sweep moves exactly the
  oracle's particles.
"""
import numpy as np
import pytest

import oracle
from sdr_b200 import _lib
from tests.gpu_common import f32, make_pair
from tests.gpu_states import sync_faces
from tests.test_oracle_kats import box_tris

pytestmark = pytest.mark.gpu


def test_sdf_staging_wait_runs_out_and_reports():
    import time

    from sdr_b200.solver import sdf_from_mesh
    tris = box_tris()
    before = sdf_from_mesh(tris, 0.5, 2.5)
    _lib.check(_lib.load().sdr_debug_inject(_lib.FAULT_SDF_STAGING))
    t0 = time.perf_counter()
    with pytest.raises(_lib.SdrError) as e:
        sdf_from_mesh(tris, 0.5, 2.5)
    waited = time.perf_counter() - t0
    assert e.value.code == _lib.SDR_ERR_DEVICE_TIMEOUT
    assert "staging wait" in str(e.value)
    assert 0.5 < waited < 30.0
    # the context is still usable and the hook was one-shot: the same field as before
    g = sdf_from_mesh(tris, 0.5, 2.5)
    assert np.array_equal(g.data.view(np.uint64), before.data.view(np.uint64))


def _checkerboard(gpu, orc):
    """24 particles in every cavity cell of even i+j+k (thousands of candidates)."""
    nx, ny, nz = gpu.grid_dims
    st = gpu.stats()
    org = np.array([st.origin.x, st.origin.y, st.origin.z])
    cav = np.flatnonzero(gpu.cavity_mask().reshape(-1))
    ijk = np.stack([cav % nx, (cav // nx) % ny, cav // (nx * ny)], axis=1)
    ijk = ijk[ijk.sum(axis=1) % 2 == 0]
    rng = np.random.default_rng(3)
    pos = org + (ijk.repeat(24, axis=0) + 0.5 + rng.uniform(-0.3, 0.3, (len(ijk) * 24, 3))) * gpu.dx
    pos = f32(pos)
    vel = np.zeros_like(pos)
    gpu.set_particles(pos, vel)
    orc.set_particles(pos, vel)
    sync_faces(gpu, orc)
    return pos


def test_candidate_list_overflow_reports_capacity_and_recovers():
    gpu, orc, res = make_pair()
    pos = _checkerboard(gpu, orc)
    gpu.set_candidate_capacity(100)
    with pytest.raises(_lib.SdrError) as e:
        gpu.run_phase(_lib.PHASE_REDISTRIBUTE)
    assert e.value.code == _lib.SDR_ERR_CAPACITY
    # nothing moved on the sweep that overflowed; the solver is still usable
    pg, _ = gpu.particles()
    assert np.array_equal(pg, pos)
    gpu.set_candidate_capacity(0)
    gpu.set_particles(pos, np.zeros_like(pos))
    gpu.run_phase(_lib.PHASE_REDISTRIBUTE)
    orc.phase(oracle.PHASE_REDISTRIBUTE)
    pg, _ = gpu.particles()
    po, _ = orc.particles()
    assert np.array_equal(np.any(pg != pos, axis=1), np.any(po != pos, axis=1))
    assert np.any(po != pos)
