"""Preview helpers on the host (src/render.rs): slice planes, the metrics
plot against the oracle's restatement, and PNG output decoded independently."""
import math
import struct
import zlib

import numpy as np
import pytest

import oracle
from sdr_b200 import _lib
from sdr_b200.render import SlicePlane, render_timeseries, save_png


def _plane(p: SlicePlane):
    d = p.as_dict()
    return (d["hax"], d["vax"], d["oax"]), bool(d["flip_v"]), bool(d["project"]), bool(d["amber"]), d["slice"], d["slab"]


def test_gravity_projection_picks_axes():  # render.rs:518-528
    axes, flip, project, amber, _, slab = _plane(SlicePlane.projected_along_gravity((0.0, 8.0, -6.0)))
    assert axes == (2, 1, 0)
    assert project and amber and math.isinf(slab)
    assert not flip  # +gravity along +y maps downward


def _gravity_restated(g):
    ga = [abs(x) for x in g]
    oax = min(range(3), key=lambda a: ga[a])  # first minimum
    rem = [a for a in range(3) if a != oax]
    vax, hax = (rem[0], rem[1]) if ga[rem[0]] >= ga[rem[1]] else (rem[1], rem[0])
    return (hax, vax, oax), g[vax] < 0


@pytest.mark.parametrize("g", [(0.0, -9.81, 0.0), (0.0, 8.03, -5.63), (0.0, 0.0, -9.81), (3.0, -3.0, 3.0),
                               (-1.0, 0.5, 0.25), (0.0, 0.0, 0.0)])
def test_gravity_projection_matches_restatement(g):
    axes, flip, *_ = _plane(SlicePlane.projected_along_gravity(g))
    assert (axes, flip) == _gravity_restated(g)


def test_fixed_planes():  # render.rs:64-103
    assert _plane(SlicePlane.xy(0.01, 0.002)) == ((0, 1, 2), True, False, False, 0.01, 0.002)
    assert _plane(SlicePlane.xz(0.01, 0.002)) == ((0, 2, 1), False, False, False, 0.01, 0.002)
    assert _plane(SlicePlane.yz(0.01, 0.002)) == ((1, 2, 0), True, False, False, 0.01, 0.002)


def _frames(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        f = {k: (i if t is not C_DOUBLE else float(rng.uniform(-0.2, 1.3))) for k, t in _lib.FrameMetricsC._fields_}
        f["peak_wall_pressure_pa"] = float(rng.uniform(0, 5e4))
        out.append(f)
    return out


C_DOUBLE = _lib.FrameMetricsC._fields_[1][1]


@pytest.mark.parametrize("n,w,h", [(0, 400, 200), (1, 400, 200), (2, 400, 200), (5, 400, 200), (18, 720, 360),
                                   (300, 97, 41)])
def test_timeseries_matches_oracle(n, w, h):
    frames = _frames(n, n + w)
    got = render_timeseries(frames, w, h)
    ref = oracle.render_timeseries(frames, w, h)
    assert got.shape == (h, w, 3)  # render.rs:583-585
    assert np.array_equal(got, ref)


def _read_png(path):
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, chunks = 8, []
    while pos < len(data):
        (n,) = struct.unpack(">I", data[pos:pos + 4])
        typ = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        (crc,) = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])
        assert crc == zlib.crc32(typ + body)
        chunks.append((typ, body))
        pos += 12 + n
    assert chunks[0][0] == b"IHDR" and chunks[-1][0] == b"IEND"
    w, h, depth, ctype, comp, filt, lace = struct.unpack(">IIBBBBB", chunks[0][1])
    assert (depth, ctype, comp, filt, lace) == (8, 2, 0, 0, 0)
    raw = zlib.decompress(b"".join(b for t, b in chunks if t == b"IDAT"))
    rows = np.frombuffer(raw, dtype=np.uint8).reshape(h, 1 + 3 * w)
    assert not rows[:, 0].any()  # filter type 0 on every row
    return rows[:, 1:].reshape(h, w, 3)


def test_png_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    for shape in [(1, 1, 3), (37, 53, 3), (200, 300, 3)]:
        img = rng.integers(0, 256, shape, dtype=np.uint8)
        p = tmp_path / f"img_{shape[0]}.png"
        save_png(img, p)
        assert np.array_equal(_read_png(p), img)
    with pytest.raises(RuntimeError):
        save_png(img, tmp_path / "missing" / "x.png")


def test_oracle_renderer_passes_the_reference_render_tests():
    """The oracle's restatement of render.rs, pinned by the reference's own
    render tests (render.rs:492-566) on their short_run scene: the slice shows
    cavity interior and coloured fluid/needle pixels, the gravity projection a
    silhouette and an amber pool, and the amber render is deterministic."""
    from sdr_b200 import scene as sc
    from tests.helpers import oracle_solver
    toml = ("[sim]\nresolution_mm = 2.5\nduration_s = 0.05\nframes = 5\n"
            "[needle]\nauto = true\ndiameter_mm = 1.2\nflow_rate_ml_s = 6.0\n"
            "[fluid]\nparticles_per_cell = 16\n")
    res = sc.SceneConfig.from_toml_str(toml).resolve()
    orc = oracle_solver(res)
    for _ in range(res.frames):
        orc.step(res.frame_dt)
    interior = np.array([232, 236, 244], dtype=np.uint8)

    def coloured(img):
        return bool(((img.max(axis=2).astype(int) - img.min(axis=2).astype(int)) > 60).any())

    xy = SlicePlane.xy(res.needle.tip[2], res.sim_dx).as_dict()
    img = orc.render_slice(xy, 300, 0.0)
    assert img.shape[0] > 0 and img.shape[1] > 0
    assert (img == interior).all(axis=2).any(), "no cavity interior was drawn"
    assert coloured(img), "no fluid/needle pixels rendered"
    g = SlicePlane.projected_along_gravity(res.fluid.gravity).as_dict()
    a = orc.render_slice(g, 300, 0.0)
    assert (a == interior).all(axis=2).any(), "no cavity silhouette"
    assert coloured(a)
    r, gg, b = (a[..., k].astype(int) for k in range(3))
    assert ((r > gg) & (gg > b) & ((r - b) > 20)).any(), "no amber fluid pool was rendered"
    assert np.array_equal(a, orc.render_slice(g, 300, 0.0)), "amber render is not deterministic"
