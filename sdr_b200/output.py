"""Frame output (``src/output.rs``): VTK / XYZ particle files and frame names.

``write_points`` and ``frame_path`` mirror ``write_points_vtk``,
``write_points_xyz`` and ``frame_path``; ``FrameWriter`` is the per-frame
output of ``cmd_simulate`` (``src/main.rs:255-266``) done in the background:
the positions are copied off the device on the solver's stream and written by
a library thread while the next frames run.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import FORMAT_VTK, FORMAT_XYZ, check  # noqa: F401

_FORMATS = {"vtk": FORMAT_VTK, "xyz": FORMAT_XYZ}


def _fmt(fmt) -> int:
    return _FORMATS[fmt] if isinstance(fmt, str) else int(fmt)


def write_points(path: str, xyz: np.ndarray, fmt="vtk") -> None:
    """Positions (n x 3, stored as f32 like the device) to a VTK or XYZ file."""
    a = np.ascontiguousarray(np.asarray(xyz, dtype=np.float32).reshape(-1, 3))
    check(_lib.load().sdr_write_points(str(path).encode(), _fmt(fmt), a.ctypes.data_as(C.POINTER(C.c_float)),
                                       a.shape[0]))


def frame_path(dir: str, prefix: str, frame: int, fmt="vtk") -> str:
    buf = C.create_string_buffer(4096)
    check(_lib.load().sdr_frame_path(str(dir).encode(), prefix.encode(), int(frame), _fmt(fmt), buf, 4096))
    return buf.value.decode()


class FrameWriter:
    """Double-buffered asynchronous frame output; ``dir`` must exist."""

    def __init__(self, dir: str, prefix: str = "particles", fmt="vtk"):
        self._L = _lib.load()
        h = C.c_void_p()
        check(self._L.sdr_frame_writer_create(str(dir).encode(), prefix.encode(), _fmt(fmt), C.byref(h)))
        self._h = h

    def submit(self, solver, frame: int) -> None:
        check(self._L.sdr_frame_writer_submit(self._h, solver._h, int(frame)))

    def flush(self) -> None:
        check(self._L.sdr_frame_writer_flush(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            h, self._h = self._h, None
            check(self._L.sdr_frame_writer_destroy(h))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
