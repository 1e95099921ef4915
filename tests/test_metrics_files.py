"""metrics.json / metrics.csv / summary.json (src/metrics.rs:385-431,
src/main.rs:306-310) through the C ABI, on the CPU.

The expected text is built here from a restatement of the two number formats
the reference uses: serde_json's f64 (shortest round-trip digits; plain with at
least one fractional digit for 1e-5 <= |v| < 1e16, else d.ddde[-]x; null when
not finite) and Rust's `{}` for f64 (shortest digits, plain notation, no
exponent). The shortest digits come from Python's repr, an independent
implementation of the same shortest round-trip rule. The reference's own test
(`writes_json_and_csv`, metrics.rs:553-576) only checks for a field name and
the CSV line count; it is repeated here.
"""
import ctypes as C
import json
import math
from decimal import Decimal

import numpy as np
import pytest

from sdr_b200 import _lib

FRAME_KEYS = [n for n, _ in _lib.FrameMetricsC._fields_]
SUMMARY_KEYS = [n for n, _ in _lib.SummaryC._fields_]
INT_KEYS = {"frame", "particles", "membrane_artifacts", "pcg_iters", "frames", "membrane_artifacts_total"}


def _shortest(v: float):
    """Shortest round-trip decimal digits of |v| and k with |v| = digits * 10**k."""
    _, digs, exp = Decimal(repr(abs(v))).as_tuple()
    digs = list(digs)
    while len(digs) > 1 and digs[-1] == 0:
        digs.pop()
        exp += 1
    return "".join(map(str, digs)), exp


def serde_f64(v: float) -> str:
    if not math.isfinite(v):
        return "null"
    sign = "-" if math.copysign(1.0, v) < 0 else ""
    if v == 0:
        return sign + "0.0"
    d, k = _shortest(v)
    n = len(d)
    kk = n + k
    if k >= 0 and kk <= 16:
        body = d + "0" * k + ".0"
    elif 0 < kk <= 16:
        body = d[:kk] + "." + d[kk:]
    elif -5 < kk <= 0:
        body = "0." + "0" * (-kk) + d
    else:
        body = d[0] + ("." + d[1:] if n > 1 else "") + "e" + str(kk - 1)
    return sign + body


def rust_display_f64(v: float) -> str:
    if math.isnan(v):
        return "NaN"
    if math.isinf(v):
        return "inf" if v > 0 else "-inf"
    sign = "-" if math.copysign(1.0, v) < 0 else ""
    if v == 0:
        return sign + "0"
    d, k = _shortest(v)
    n = len(d)
    if k >= 0:
        body = d + "0" * k
    elif -k < n:
        body = d[:n + k] + "." + d[n + k:]
    else:
        body = "0." + "0" * (-k - n) + d
    return sign + body


def _json_object(rec: dict, keys, ind: str) -> str:
    lines = [f'{ind}  "{k}": {rec[k] if k in INT_KEYS else serde_f64(rec[k])}' for k in keys]
    return "{\n" + ",\n".join(lines) + "\n" + ind + "}"


def expected_frames_json(frames) -> str:
    if not frames:
        return "[]"
    return "[\n" + ",\n".join("  " + _json_object(f, FRAME_KEYS, "  ") for f in frames) + "\n]"


def expected_frames_csv(frames) -> str:
    rows = [",".join(FRAME_KEYS)]
    for f in frames:
        rows.append(",".join(str(f[k]) if k in INT_KEYS else rust_display_f64(f[k]) for k in FRAME_KEYS))
    return "\n".join(rows) + "\n"


SPECIAL = [0.0, -0.0, 1.0, -1.0, 0.1, 0.5, 2.5, 100.0, 1e-5, 9.999e-6, 1e-6, 1.5e-7, 123.456, 1e15, 1e16,
           9.999999999999998e15, 1.2345678901234567e16, 123456789012345680.0, 5e-324, 2.2250738585072014e-308,
           1.7976931348623157e308, 0.30000000000000004, 1 / 3, 2.0 ** 53, 1e21, 1e22, 1e100, -7.25e-9,
           float("nan"), float("inf"), float("-inf")]


def _values(rng, n):
    mags = 10.0 ** rng.uniform(-12, 22, n)
    vals = list(np.where(rng.random(n) < 0.5, -1.0, 1.0) * mags * rng.random(n))
    vals += [float(np.float32(x)) for x in rng.standard_normal(n // 4)]  # f32-valued quantities
    return [float(v) for v in vals] + SPECIAL


def _frames(vals, rng):
    out = []
    for i in range(0, len(vals), 13):
        chunk = (vals[i:i + 13] + SPECIAL)[:13]
        rec, it = {}, iter(chunk)
        for k in FRAME_KEYS:
            rec[k] = int(rng.integers(0, 2 ** 40)) if k in INT_KEYS else next(it)
        out.append(rec)
    return out


def _frames_c(frames):
    arr = (_lib.FrameMetricsC * max(len(frames), 1))()
    for i, f in enumerate(frames):
        for k in FRAME_KEYS:
            setattr(arr[i], k, f[k])
    return arr


@pytest.fixture(scope="module")
def L():
    return _lib.load()


def test_frames_json_and_csv_match_reference_formats(L, tmp_path):
    rng = np.random.default_rng(11)
    frames = _frames(_values(rng, 4000), rng)
    arr = _frames_c(frames)
    pj, pc = tmp_path / "metrics.json", tmp_path / "metrics.csv"
    assert L.sdr_frames_write_json(arr, len(frames), str(pj).encode()) == 0
    assert L.sdr_frames_write_csv(arr, len(frames), str(pc).encode()) == 0
    got_j, got_c = pj.read_text(), pc.read_text()
    assert got_j == expected_frames_json(frames)
    assert got_c == expected_frames_csv(frames)
    # the JSON reads back to the same numbers (non-finite values as null)
    back = json.loads(got_j)
    for f, b in zip(frames, back):
        for k in FRAME_KEYS:
            v = f[k]
            if k not in INT_KEYS and not math.isfinite(v):
                assert b[k] is None
            else:
                assert b[k] == v and (k in INT_KEYS or math.copysign(1, b[k]) == math.copysign(1, v))


def test_summary_json(L, tmp_path):
    rng = np.random.default_rng(12)
    vals = _values(rng, 64)
    sm = _lib.SummaryC()
    rec = {}
    for i, k in enumerate(SUMMARY_KEYS):
        rec[k] = int(rng.integers(0, 1000)) if k in INT_KEYS else vals[i]
        setattr(sm, k, rec[k])
    p = tmp_path / "summary.json"
    assert L.sdr_summary_write_json(C.byref(sm), str(p).encode()) == 0
    assert p.read_text() == _json_object(rec, SUMMARY_KEYS, "")


def test_reference_writes_json_and_csv_checks(L, tmp_path):
    """metrics.rs:553-576: the JSON names fill_fraction, the CSV has a header and one line per frame."""
    frames = _frames(SPECIAL, np.random.default_rng(1))[:2]
    arr = _frames_c(frames)
    pj, pc = tmp_path / "m.json", tmp_path / "m.csv"
    assert L.sdr_frames_write_json(arr, 2, str(pj).encode()) == 0
    assert L.sdr_frames_write_csv(arr, 2, str(pc).encode()) == 0
    assert "fill_fraction" in pj.read_text()
    assert len(pc.read_text().splitlines()) >= 3


def test_empty_history_and_io_errors(L, tmp_path):
    arr = _frames_c([])
    pj, pc = tmp_path / "e.json", tmp_path / "e.csv"
    assert L.sdr_frames_write_json(arr, 0, str(pj).encode()) == 0
    assert L.sdr_frames_write_csv(arr, 0, str(pc).encode()) == 0
    assert pj.read_text() == "[]"
    assert pc.read_text() == ",".join(FRAME_KEYS) + "\n"
    bad = str(tmp_path / "missing" / "x.json").encode()
    assert L.sdr_frames_write_json(arr, 0, bad) == _lib.SDR_ERR_IO
    assert b"missing" in L.sdr_last_error()
    assert L.sdr_summary_write_json(None, bad) == _lib.SDR_ERR_INVALID
