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
