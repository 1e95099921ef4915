"""The winding-number SDF at the real-cavity workload's scale: the perturbed
ellipsoid of 20,480 triangles voxelised at 0.5 mm (65k nodes, 1.3e9
node-triangle pairs) on the device, checked bit for bit against the oracle's
Sdf::from_mesh node rule (sdf.rs:53-86, 187-205) at 3000 nodes: every node
within two cells of the surface that a seeded draw picks, and as many drawn
uniformly (the oracle evaluates single nodes; the whole grid would take it
about a minute)."""
import numpy as np
import pytest

import oracle
from sdr_b200 import workloads
from tests.gpu_common import record

pytestmark = pytest.mark.gpu


def test_sdf_mesh_real_cavity_scale_bit_exact():
    from sdr_b200.solver import sdf_from_mesh
    w = workloads.real_cavity(seed=2)
    tris = np.ascontiguousarray(w.tris, dtype=np.float64)
    dx, pad = w.res.sdf_dx, w.res.mesh_padding
    g = sdf_from_mesh(tris, dx, pad)
    origin, dims = oracle.sdf_mesh_grid(tris, dx, pad)
    nx, ny, nz = dims
    assert g.data.shape == (nz, ny, nx)
    assert np.array_equal(np.asarray(g.origin, dtype=np.float64), origin)
    rng = np.random.default_rng(11)
    flat = g.data.reshape(-1)
    near = np.flatnonzero(np.abs(flat) < 2.0 * dx)
    pick = np.concatenate([rng.choice(near, size=min(1500, len(near)), replace=False),
                           rng.choice(flat.size, size=1500, replace=False)])
    mism = 0
    sign_mism = 0
    for c in pick:
        i, j, k = c % nx, (c // nx) % ny, c // (nx * ny)
        p = origin + np.array([i * dx, j * dx, k * dx])
        ref = oracle.signed_distance_to_mesh(p, tris)
        mism += int(np.float64(ref).view(np.uint64) != flat[c].view(np.uint64))
        sign_mism += int((ref < 0) != (flat[c] < 0))
    record("sdf_mesh_real_cavity", {"tris": int(len(tris)), "nodes": int(flat.size), "checked": int(len(pick)),
                                    "near_surface": int(min(1500, len(near))), "bit_mismatch": mism,
                                    "sign_mismatch": sign_mism, "inside": int((flat < 0).sum())})
    assert sign_mism == 0
    assert mism == 0
