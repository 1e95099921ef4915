"""Frame output against the reference's own output tests (src/output.rs:125-185)
and its number formatting (Rust `{}` for f64: shortest round-trip digits in
fixed notation)."""
from decimal import Decimal
import math
import struct

import numpy as np
import pytest

from sdr_b200 import _lib
from sdr_b200.output import frame_path, write_points


def rust_display(x: float) -> str:
    """Rust's Display for f64, restated: Python's repr has the same shortest
    round-trip digits; print them without an exponent and without '.0'."""
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "inf" if x > 0 else "-inf"
    if x == 0.0:
        return "-0" if math.copysign(1.0, x) < 0 else "0"
    s = format(Decimal(repr(x)), "f")
    if "." in s:
        s = s.rstrip("0").rstrip(".")
    return s


def read_vtk(path):
    """read_points_vtk (output.rs:55-95): the POINTS block as f64."""
    toks = open(path).read().split()
    i = toks.index("POINTS")
    n = int(toks[i + 1])
    vals = [float(t) for t in toks[i + 3:i + 3 + 3 * n]]
    return np.array(vals).reshape(n, 3)


def test_vtk_has_expected_structure(tmp_path):  # output.rs:132-144
    p = tmp_path / "pts.vtk"
    write_points(p, [[0.0, 1.0, 2.0], [-1.0, 0.5, 3.0]])
    text = p.read_text()
    assert "DATASET UNSTRUCTURED_GRID" in text
    assert "POINTS 2 double" in text
    assert "0 1 2" in text
    assert "CELL_TYPES 2" in text
    assert text.startswith("# vtk DataFile Version 4.2\nsdr irrigation particles\nASCII\n")
    assert "CELLS 2 4\n1 0\n1 1\nCELL_TYPES 2\n1\n1\n" in text


def test_vtk_round_trips_positions(tmp_path):  # output.rs:146-163
    pts = np.array([[0.0, 1.0, 2.0], [-1.5, 0.25, 3.5], [10.0, -20.0, 30.0]])
    p = tmp_path / "rt.vtk"
    write_points(p, pts)
    assert np.array_equal(read_vtk(p), pts)


def test_vtk_numbers_are_rust_f64_display_of_the_f32_values(tmp_path):
    rng = np.random.default_rng(3)
    pts = np.concatenate([rng.standard_normal((200, 3)) * 0.02,
                          np.array([[1e-7, -0.0, 0.0], [123456.75, 3.4e-30, -2.5e10]])]).astype(np.float32)
    p = tmp_path / "f.vtk"
    write_points(p, pts)
    lines = p.read_text().splitlines()
    body = lines[5:5 + len(pts)]
    expect = [" ".join(rust_display(float(v)) for v in row) for row in pts]
    assert body == expect
    assert np.array_equal(read_vtk(p), pts.astype(np.float64))  # widened f32 round-trips exactly


def test_xyz_is_binary_f32_triples(tmp_path):  # output.rs:165-178
    p = tmp_path / "pts.xyz"
    write_points(p, [[0.0, 1.0, 2.0], [3.0, 4.0, 5.0]], fmt="xyz")
    b = p.read_bytes()
    assert len(b) == 2 * 12
    assert struct.unpack("<f", b[0:4])[0] == 0.0
    assert struct.unpack("<f", b[16:20])[0] == 4.0


def test_frame_path_is_zero_padded():  # output.rs:180-184
    assert frame_path("/tmp/out", "particles", 42, "vtk").endswith("particles_000042.vtk")
    assert frame_path("out/", "p", 1234567, "xyz") == "out/p_1234567.xyz"


def test_unwritable_path_reports_io_error(tmp_path):
    with pytest.raises(_lib.SdrError, match="creating"):
        write_points(tmp_path / "missing_dir" / "x.vtk", [[0.0, 0.0, 0.0]])
