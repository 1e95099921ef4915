"""The no-allocation SDF entry point against the allocating one.

sdr_sdf_from_mesh_noalloc serves callers that cannot allocate device memory
(a fixed device-memory budget handed out up front, work issued during stream
capture, loops that cannot take cudaMalloc's synchronisation): it reads and
writes caller-owned device buffers and keeps its scratch in a static device
array. Both entry points run the same kernel, so their outputs must agree bit
for bit, on every call (the scratch keeps the previous call's contents).
This file is collected last so a failure here comes after every other test.
"""
import ctypes as C

import numpy as np
import pytest

from sdr_b200 import _lib
from sdr_b200.cavity import perturbed_ellipsoid

pytestmark = pytest.mark.gpu


def test_noalloc_sdf_matches_allocating_entry_point():
    import torch
    from sdr_b200.solver import sdf_from_mesh

    lib = _lib.load()
    cav = perturbed_ellipsoid(11, subdiv=3)
    dx, pad = 1.0e-3, 3.0e-3
    ref = sdf_from_mesh(cav.tris, dx, pad)  # the allocating entry point
    nz, ny, nx = ref.data.shape
    dims = (C.c_uint64 * 3)(nx, ny, nz)
    origin = _lib.Vec3(*ref.origin)
    tris_dev = torch.tensor(np.ascontiguousarray(cav.tris), dtype=torch.float64, device="cuda")
    out_dev = torch.empty(nx * ny * nz, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        out_dev.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = lib.sdr_sdf_from_mesh_noalloc(C.c_void_p(tris_dev.data_ptr()), len(cav.tris), origin, dx, dims,
                                           C.c_void_p(out_dev.data_ptr()), C.c_void_p(stream))
        _lib.check(rc)
        got = out_dev.cpu().numpy().reshape(nz, ny, nx)
        assert np.array_equal(got.view(np.uint64), ref.data.view(np.uint64)), f"call {call} differs"


def test_noalloc_rejects_meshes_beyond_the_scratch():
    import torch
    lib = _lib.load()
    n = _lib.NOALLOC_MAX_TRIANGLES + 1
    tris_dev = torch.zeros(n * 9, dtype=torch.float64, device="cuda")
    out_dev = torch.empty(8, dtype=torch.float64, device="cuda")
    dims = (C.c_uint64 * 3)(2, 2, 2)
    rc = lib.sdr_sdf_from_mesh_noalloc(C.c_void_p(tris_dev.data_ptr()), n, _lib.Vec3(0, 0, 0), 1.0, dims,
                                       C.c_void_p(out_dev.data_ptr()), None)
    assert rc == 1
    assert b"scratch holds" in lib.sdr_last_error()
