"""Asynchronous frame output: the files the background writer produces are
byte-identical to synchronous writes of the same frames' positions."""
import pytest

from sdr_b200 import scene as sc
from sdr_b200.output import FrameWriter, frame_path, write_points
from tests.gpu_common import SMOKE_TOML

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fmt", ["vtk", "xyz"])
def test_frame_writer_matches_synchronous_writes(tmp_path, fmt):
    from sdr_b200.solver import build_scene
    b = build_scene(sc.SceneConfig.from_toml_str(SMOKE_TOML))
    d_async, d_sync = tmp_path / "async", tmp_path / "sync"
    d_async.mkdir()
    d_sync.mkdir()
    with FrameWriter(d_async, "particles", fmt) as w:
        for f in range(3):
            b.solver.step(b.frame_dt)
            w.submit(b.solver, f)          # returns before the file is written
            pos, _ = b.solver.particles_f32()
            write_points(frame_path(d_sync, "particles", f, fmt), pos, fmt)
        w.flush()
    for f in range(3):
        a = open(frame_path(d_async, "particles", f, fmt), "rb").read()
        s = open(frame_path(d_sync, "particles", f, fmt), "rb").read()
        assert a == s and len(a) > 0


def test_metrics_files_from_a_run(tmp_path):
    """metrics.json / metrics.csv written from a collector after a short run
    equal the same writers on the recorded frames; summary.json reads back as
    the summary."""
    import ctypes as C
    import json

    from sdr_b200 import _lib
    from sdr_b200.solver import MetricsCollector, build_scene
    b = build_scene(sc.SceneConfig.from_toml_str(SMOKE_TOML))
    m = MetricsCollector(b.solver, b.cavity_volume)
    for f in range(3):
        b.solver.step(b.frame_dt)
        m.record(b.solver, f)
    m.write_json(tmp_path / "metrics.json")
    m.write_csv(tmp_path / "metrics.csv")
    m.write_summary_json(tmp_path / "summary.json")
    arr = (_lib.FrameMetricsC * 3)()
    for i, rec in enumerate(m.history):
        for k, v in rec.items():
            setattr(arr[i], k, v)
    L = _lib.load()
    assert L.sdr_frames_write_json(arr, 3, str(tmp_path / "f.json").encode()) == 0
    assert L.sdr_frames_write_csv(arr, 3, str(tmp_path / "f.csv").encode()) == 0
    assert (tmp_path / "metrics.json").read_bytes() == (tmp_path / "f.json").read_bytes()
    assert (tmp_path / "metrics.csv").read_bytes() == (tmp_path / "f.csv").read_bytes()
    frames = json.loads((tmp_path / "metrics.json").read_text())
    assert [f["frame"] for f in frames] == [0, 1, 2] and frames[2]["particles"] == m.history[2]["particles"]
    assert json.loads((tmp_path / "summary.json").read_text()) == m.summary()


def _read_vtk_points(path):
    """POINTS block of a legacy ASCII VTK file (read_points_vtk, output.rs:57-96)."""
    import numpy as np
    lines = open(path).read().split("\n")
    i = next(k for k, l in enumerate(lines) if l.startswith("POINTS"))
    n = int(lines[i].split()[1])
    vals = " ".join(lines[i + 1:]).split()[: 3 * n]
    return np.array([float(v) for v in vals]).reshape(n, 3)


def test_frame_files_hold_the_solver_state(tmp_path):
    """The background writer's frames against the solver's own particle
    state, read back independently: VTK text parses back to the stored f32
    positions bit for bit (shortest round-trip digits, output.rs:23-48), XYZ
    bytes are those f32 values (output.rs:98-110)."""
    import numpy as np
    from sdr_b200.solver import build_scene
    b = build_scene(sc.SceneConfig.from_toml_str(SMOKE_TOML))
    for fmt in ("vtk", "xyz"):
        d = tmp_path / fmt
        d.mkdir()
        with FrameWriter(d, "particles", fmt) as w:
            b.solver.step(b.frame_dt)
            w.submit(b.solver, 7)
            w.flush()
        pos32, _ = b.solver.particles_f32()
        path = frame_path(d, "particles", 7, fmt)
        if fmt == "vtk":
            back = _read_vtk_points(path)
            assert back.shape == pos32.shape and len(back) > 0
            assert np.array_equal(back, pos32.astype(np.float64))
        else:
            raw = np.fromfile(path, dtype="<f4").reshape(-1, 3)
            assert np.array_equal(raw.view(np.uint32), np.ascontiguousarray(pos32, dtype=np.float32).view(np.uint32))
