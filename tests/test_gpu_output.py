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
