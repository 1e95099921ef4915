"""The no-allocation SDF entry point against the allocating one.

sdr_sdf_from_mesh_noalloc serves callers that cannot allocate device memory
(a process that carves its whole device-memory budget into a pool at start-up
and must not grow it, loops that cannot take cudaMalloc's synchronisation): it
reads and writes caller-owned device buffers and keeps its scratch in a static
device array. Both entry points run the same kernel, so their outputs must
agree bit for bit on every call, including a smaller mesh after a larger one
(the scratch keeps the previous call's contents, and the padding of the last
staging tile must be cleared again). Free device memory does not change
across the calls. This file is collected last so a failure here comes after
every other test.
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
    dx, pad = 1.0e-3, 3.0e-3
    # a mesh of whole staging tiles (1280 triangles), then a smaller ragged one (320)
    meshes = [perturbed_ellipsoid(11, subdiv=3), perturbed_ellipsoid(12, subdiv=2)]
    assert len(meshes[0].tris) % 128 == 0 and len(meshes[1].tris) % 128 != 0
    refs = [sdf_from_mesh(m.tris, dx, pad) for m in meshes]  # the allocating entry point
    stream = torch.cuda.current_stream().cuda_stream
    bufs = []
    for m, ref in zip(meshes, refs):
        nz, ny, nx = ref.data.shape
        bufs.append((torch.tensor(np.ascontiguousarray(m.tris), dtype=torch.float64, device="cuda"),
                     torch.empty(nx * ny * nz, dtype=torch.float64, device="cuda")))
    torch.cuda.synchronize()
    free0 = alloc0 = None
    # call 0 does the first-call set-up (the scratch address lookup); free
    # memory is taken after it and must not move over the calls that follow
    for call, k in enumerate([0, 0, 1, 0, 1]):
        ref, (tris_dev, out_dev) = refs[k], bufs[k]
        nz, ny, nx = ref.data.shape
        dims = (C.c_uint64 * 3)(nx, ny, nz)
        out_dev.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = lib.sdr_sdf_from_mesh_noalloc(C.c_void_p(tris_dev.data_ptr()), len(meshes[k].tris), _lib.Vec3(*ref.origin),
                                           dx, dims, C.c_void_p(out_dev.data_ptr()), C.c_void_p(stream))
        _lib.check(rc)
        got = out_dev.cpu().numpy().reshape(nz, ny, nx)
        assert np.array_equal(got.view(np.uint64), ref.data.view(np.uint64)), f"call {call} (mesh {k}) differs"
        if call == 0:
            free0, alloc0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_allocated()
        else:
            assert torch.cuda.mem_get_info()[0] == free0, f"call {call} changed free device memory"
            assert torch.cuda.memory_allocated() == alloc0


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
