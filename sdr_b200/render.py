"""Previews (``src/render.rs``): slice and gravity-projection images of a
solver's state drawn on the device, the metrics plot, and PNG output.

``SlicePlane`` mirrors the reference's constructors (``xy``, ``xz``, ``yz``,
``projected_along_gravity``); ``render_slice`` returns an ``(h, w, 3)`` uint8
image equal to the reference's ``render_slice`` for the same particle state.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _lib
from ._lib import check

_U8P = C.POINTER(C.c_uint8)


class SlicePlane:
    """SlicePlane (render.rs:45-136)."""

    def __init__(self, c: _lib.SlicePlaneC):
        self.c = c

    @classmethod
    def _make(cls, fn, *args) -> "SlicePlane":
        c = _lib.SlicePlaneC()
        check(fn(*args, C.byref(c)))
        return cls(c)

    @classmethod
    def xy(cls, slice_: float, slab: float) -> "SlicePlane":
        return cls._make(_lib.load().sdr_slice_plane_xy, float(slice_), float(slab))

    @classmethod
    def xz(cls, slice_: float, slab: float) -> "SlicePlane":
        return cls._make(_lib.load().sdr_slice_plane_xz, float(slice_), float(slab))

    @classmethod
    def yz(cls, slice_: float, slab: float) -> "SlicePlane":
        return cls._make(_lib.load().sdr_slice_plane_yz, float(slice_), float(slab))

    @classmethod
    def projected_along_gravity(cls, gravity) -> "SlicePlane":
        g = _lib.Vec3(*(float(x) for x in gravity))
        return cls._make(_lib.load().sdr_slice_plane_gravity, g)

    def as_dict(self) -> dict:
        return {n: getattr(self.c, n) for n, _ in self.c._fields_}


def render_slice(solver, plane: SlicePlane, target_px: int = 600, vmax: float = 0.0) -> np.ndarray:
    """render_slice (render.rs:139-236) of the solver's current state."""
    L = _lib.load()
    w, h = C.c_uint32(), C.c_uint32()
    rc = L.sdr_render_slice(solver._h, C.byref(plane.c), int(target_px), float(vmax), None, 0, C.byref(w),
                            C.byref(h))
    if rc != _lib.SDR_ERR_BUFFER:
        check(rc)
    img = np.zeros((h.value, w.value, 3), dtype=np.uint8)
    check(L.sdr_render_slice(solver._h, C.byref(plane.c), int(target_px), float(vmax), img.ctypes.data_as(_U8P),
                             img.nbytes, C.byref(w), C.byref(h)))
    return img


def render_timeseries(frames: Sequence[dict], width: int = 720, height: int = 360) -> np.ndarray:
    """render_timeseries (render.rs:351-406); frames are FrameMetrics dicts."""
    arr = (_lib.FrameMetricsC * max(len(frames), 1))()
    for i, f in enumerate(frames):
        for k, _ in _lib.FrameMetricsC._fields_:
            setattr(arr[i], k, f[k])
    img = np.zeros((int(height), int(width), 3), dtype=np.uint8)
    check(_lib.load().sdr_render_timeseries(arr, len(frames), int(width), int(height), img.ctypes.data_as(_U8P),
                                            img.nbytes))
    return img


def save_png(img: np.ndarray, path) -> None:
    """save_png (render.rs:409-414)."""
    a = np.ascontiguousarray(img, dtype=np.uint8)
    if a.ndim != 3 or a.shape[2] != 3:
        raise ValueError("expected an (h, w, 3) uint8 image")
    check(_lib.load().sdr_write_png(str(path).encode(), a.ctypes.data_as(_U8P), a.shape[1], a.shape[0]))
