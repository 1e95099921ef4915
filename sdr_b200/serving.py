"""Many scenes on one GPU: batches and a request loop (``sdr_batch_*``, ``sdr_server_*``).

The reference simulates one scene per ``sdr simulate`` process
(``src/main.rs:215-386``: build the scene, ``Solver::step`` per frame,
``MetricsCollector::record``, the summary). ``run_batch`` runs that loop for
many scenes at once and ``Server`` admits scenes as they arrive, both inside
``libsdr_gpu.so``: every scene gets its own solver, CUDA stream and host
thread, and a scene's result is the same alone and beside others.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import check
from .scene import FluidParams, Needle, SolveParams
from .solver import Sdf, _dp, _v3


@dataclass
class SceneSpec:
    """One scene: ``Solver::new`` inputs plus the run length and the cavity volume."""
    sdf: Sdf
    sim_dx: float
    fluid: FluidParams
    needle: Needle
    solve: SolveParams
    cavity_volume: float
    frame_dt: float
    frames: int
    outlet: Optional[tuple] = None  # ((x0, y0, z0), (x1, y1, z1))
    max_particles: int = 0


class _Desc:
    """A SceneDesc and the arrays it points into."""

    def __init__(self, spec: SceneSpec):
        self.data = np.ascontiguousarray(spec.sdf.data, dtype=np.float64)
        nx, ny, nz = spec.sdf.dims
        f, n = spec.fluid, spec.needle
        self.c = _lib.SceneDesc()
        self.c.sdf = _lib.SdfDesc(_v3(spec.sdf.origin), spec.sdf.dx, nx, ny, nz, _dp(self.data))
        self.c.sim_dx = spec.sim_dx
        self.c.fluid = _lib.FluidParamsC(f.density, _v3(f.gravity), f.flip_ratio, int(f.particles_per_cell),
                                         f.volume_stiffness, 1 if f.redistribute else 0, 0, f.redist_cap_factor)
        self.c.needle = _lib.NeedleC(_v3(n.tip), _v3(n.axis), n.radius, n.flow_rate, n.inject_until)
        self.c.solve = _lib.SolveParamsC(int(spec.solve.max_iters), spec.solve.tol)
        if spec.outlet is not None:
            self.c.has_outlet = 1
            self.c.outlet = _lib.Aabb(_v3(spec.outlet[0]), _v3(spec.outlet[1]))
        self.c.cavity_volume = spec.cavity_volume
        self.c.frame_dt = spec.frame_dt
        self.c.frames = int(spec.frames)
        self.c.max_particles = int(spec.max_particles)


def footprint(spec: SceneSpec) -> int:
    """Device bytes the scene needs while it runs (the server's admission estimate)."""
    d = _Desc(spec)
    out = C.c_uint64()
    check(_lib.load().sdr_scene_footprint(C.byref(d.c), C.byref(out)))
    return int(out.value)


@dataclass
class SceneResult:
    status: int
    summary: Optional[dict]
    stats: Optional[dict]
    seconds: float
    error: str


def run_batch(specs: Sequence[SceneSpec], concurrency: int = 0, device: int = -1, packed: bool = False,
              counters: Optional[dict] = None) -> List[SceneResult]:
    """Run every scene to its frame count, ``concurrency`` at a time (0 = all,
    1 = one after another), or all packed into one launch per substep
    operation (``packed``, sdr_batch_run_packed); results in input order.
    ``counters`` receives the packed run's launches and packed steps."""
    L = _lib.load()
    descs = [_Desc(s) for s in specs]
    arr = (_lib.SceneDesc * len(descs))(*[d.c for d in descs])
    h = C.c_void_p()
    check(L.sdr_batch_create(arr, len(descs), int(device), C.byref(h)))
    try:
        if packed:
            check(L.sdr_batch_run_packed(h))
            if counters is not None:
                la, stp, cap, ctas = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_int32()
                check(L.sdr_batch_packed_counters(h, C.byref(la), C.byref(stp), C.byref(cap), C.byref(ctas)))
                counters.update(launches=la.value, steps=stp.value, graph_captures=cap.value,
                                ctas_per_sm=ctas.value)
        else:
            check(L.sdr_batch_run(h, int(concurrency)))
        out = []
        for i in range(len(descs)):
            st = C.c_int32()
            sm = _lib.SummaryC()
            stats = _lib.SolverStats()
            secs = C.c_double()
            err = C.create_string_buffer(512)
            check(L.sdr_batch_result(h, i, C.byref(st), C.byref(sm), C.byref(stats), C.byref(secs), err, 512))
            ok = st.value == _lib.SDR_OK
            out.append(SceneResult(st.value, sm.to_dict() if ok else None,
                                   {n: getattr(stats, n) for n, _ in stats._fields_} if ok else None,
                                   secs.value, err.value.decode()))
        return out
    finally:
        L.sdr_batch_destroy(h)


class Server:
    """Continuous batching: scenes submitted at any time run as soon as their
    footprint fits ``budget_bytes`` and one of ``max_active`` slots is free."""

    def __init__(self, budget_bytes: int, max_active: int, device: int = -1, packed: bool = False):
        self._L = _lib.load()
        h = C.c_void_p()
        create = self._L.sdr_server_create_packed if packed else self._L.sdr_server_create
        check(create(int(device), int(budget_bytes), int(max_active), C.byref(h)))
        self._h = h
        self._keep = {}

    def submit(self, spec: SceneSpec) -> int:
        d = _Desc(spec)
        t = C.c_uint64()
        check(self._L.sdr_server_submit(self._h, C.byref(d.c), C.byref(t)))
        return int(t.value)

    def poll(self, ticket: int) -> SceneResult:
        """status is one of _lib.REQ_*; summary and seconds (time-to-summary) when done."""
        st = C.c_int32()
        sm = _lib.SummaryC()
        secs = C.c_double()
        err = C.create_string_buffer(512)
        check(self._L.sdr_server_poll(self._h, int(ticket), C.byref(st), C.byref(sm), C.byref(secs), err, 512))
        done = st.value == _lib.REQ_DONE
        return SceneResult(st.value, sm.to_dict() if done else None, None, secs.value if done else 0.0,
                           err.value.decode())

    def wait(self, tickets: Sequence[int], timeout: float = 3600.0, interval: float = 0.01) -> List[SceneResult]:
        deadline = time.monotonic() + timeout
        while True:
            res = [self.poll(t) for t in tickets]
            if all(r.status in (_lib.REQ_DONE, _lib.REQ_FAILED) for r in res):
                return res
            if time.monotonic() > deadline:
                raise TimeoutError("requests still running")
            time.sleep(interval)

    def stats(self) -> dict:
        s = _lib.ServerStats()
        check(self._L.sdr_server_get_stats(self._h, C.byref(s)))
        return s.to_dict()

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.sdr_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
