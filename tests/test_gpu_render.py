"""render_slice on the device (render.cuh) against the oracle's restatement
of src/render.rs, pixel for pixel, on the same particle state and SDF, plus
the checks of the reference's own render tests (render.rs:492-576)."""
import numpy as np
import pytest

from sdr_b200.render import SlicePlane, render_slice
from tests.gpu_common import make_pair, record

pytestmark = pytest.mark.gpu

# render.rs:475-490 (the reference's short_run scene)
SHORT_RUN = """
[sim]
resolution_mm = 2.5
duration_s = 0.05
frames = 5
[needle]
auto = true
diameter_mm = 1.2
flow_rate_ml_s = 6.0
[fluid]
particles_per_cell = 16
"""

INTERIOR = np.array([232, 236, 244], dtype=np.uint8)


@pytest.fixture(scope="module")
def state():
    gpu, orc, res = make_pair(SHORT_RUN, warm_frames=5)
    return gpu, orc, res


def _colored(img):
    mx, mn = img.max(axis=2).astype(int), img.min(axis=2).astype(int)
    return bool(((mx - mn) > 60).any())


def _planes(res):
    tip = res.needle.tip
    dx = res.sim_dx
    return {
        "xy": SlicePlane.xy(tip[2], dx),   # render.rs:497-499
        "xz": SlicePlane.xz(tip[1], dx),
        "yz": SlicePlane.yz(tip[0], 2 * dx),
        "gravity": SlicePlane.projected_along_gravity(res.fluid.gravity),
    }


@pytest.mark.parametrize("name", ["xy", "xz", "yz", "gravity"])
@pytest.mark.parametrize("px", [300, 600])
def test_render_slice_matches_oracle(state, name, px):
    gpu, orc, res = state
    plane = _planes(res)[name]
    got = render_slice(gpu, plane, px, 0.0)
    ref = orc.render_slice(plane.as_dict(), px, 0.0)
    diff = int((got != ref).any(axis=2).sum())
    record(f"render_{name}_{px}", {"shape": list(got.shape), "pixels_differing": diff, "particles": len(gpu)})
    assert got.shape == ref.shape
    assert diff == 0
    assert (got == INTERIOR).all(axis=2).any(), "no cavity interior was drawn"
    assert _colored(got), "no fluid/needle pixels rendered"
    if plane.as_dict()["amber"]:  # render.rs:550-556
        r, g, b = (got[..., k].astype(int) for k in range(3))
        assert ((r > g) & (g > b) & ((r - b) > 20)).any(), "no amber fluid pool was rendered"


def test_render_fixed_vmax_and_determinism(state):
    gpu, orc, res = state
    plane = _planes(res)["xy"]
    a = render_slice(gpu, plane, 300, 2.0)
    assert np.array_equal(a, orc.render_slice(plane.as_dict(), 300, 2.0))
    g = _planes(res)["gravity"]
    assert np.array_equal(render_slice(gpu, g, 300), render_slice(gpu, g, 300))  # render.rs:558-565


def test_render_dense_pool_matches_oracle():
    """16 particles in every cavity cell (tiles far beyond the short-segment
    sort) plus particles off the image (beyond the margin tiles and partly
    covering the edges), random velocities: amber pool and dots match."""
    from tests.gpu_common import f32
    gpu, orc, res = make_pair(SHORT_RUN)
    nx, ny, nz = gpu.grid_dims
    dx = gpu.dx
    st = gpu.stats()
    org = np.array([st.origin.x, st.origin.y, st.origin.z])
    cav = np.flatnonzero(gpu.cavity_mask().reshape(-1))
    ijk = np.stack([cav % nx, (cav // nx) % ny, cav // (nx * ny)], axis=1)
    rng = np.random.default_rng(9)
    pos = org + (ijk.repeat(16, axis=0) + 0.5 + rng.uniform(-0.45, 0.45, (len(ijk) * 16, 3))) * dx
    span = np.array([nx, ny, nz]) * dx
    outside = org + rng.uniform(-0.3, 1.3, (500, 3)) * span  # some off the image, some near its edges
    pos = f32(np.concatenate([pos, outside]))
    vel = f32(rng.normal(0.0, 0.5, pos.shape))
    gpu.set_particles(pos, vel)
    orc.set_particles(pos, vel)
    for name, plane in _planes(res).items():
        for px in (300, 600):
            got = render_slice(gpu, plane, px, 0.0)
            ref = orc.render_slice(plane.as_dict(), px, 0.0)
            diff = int((got != ref).any(axis=2).sum())
            record(f"render_dense_{name}_{px}", {"particles": int(len(pos)), "pixels_differing": diff})
            assert diff == 0, (name, px)
