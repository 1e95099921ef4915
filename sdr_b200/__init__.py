"""sdr_b200 — a B200-native (sm_100a) FLIP/PIC substep for uselessgoddess/sdr.

The compute path is ``libsdr_gpu.so`` (C ABI: include/sdr_gpu.h), built in
tree by ``python -m sdr_b200.build``. This package is the Python mirror of the
reference's solver/metrics/scene API on top of that ABI.
"""
from .scene import (FluidParams, Needle, SceneConfig, SceneError, SinusParams, SolveParams,  # noqa: F401
                    load_mesh, load_obj, load_stl)

__all__ = ["FluidParams", "Needle", "SceneConfig", "SceneError", "SinusParams", "SolveParams",
           "load_mesh", "load_obj", "load_stl", "Solver", "MetricsCollector", "build_scene", "Sdf"]


def __getattr__(name):
    # The ctypes-backed classes load libsdr_gpu.so lazily, so configuration
    # parsing works on machines without the library.
    if name in ("Solver", "MetricsCollector", "build_scene", "Sdf", "sdf_from_mesh", "sdf_from_sinus",
                "surface_nets_volume", "build_sdf", "BuiltScene"):
        from . import solver
        return getattr(solver, name)
    raise AttributeError(name)
