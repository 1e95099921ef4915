"""Workload construction on the host: the pre-seeded pool's jitter is the
reference's hash_jitter (checked against the oracle) and its cells are the
deepest cavity cells along gravity."""
from types import SimpleNamespace

import numpy as np

import oracle
from sdr_b200 import scene as sc
from sdr_b200.workloads import hash_jitter, preseed_pool


def test_hash_jitter_matches_oracle():
    keys = [0, 1, 2, 3, 1000, 123456789, 2 ** 40 + 7, 2 ** 63 + 5, 2 ** 64 - 1]
    got = hash_jitter(np.array(keys, dtype=np.uint64))
    for k, row in zip(keys, got):
        assert np.array_equal(row, oracle.hash_jitter(k)), k
    assert np.all(got >= -0.3) and np.all(got < 0.3)


class _FakeSolver:
    def __init__(self, mask, dx=1e-3, origin=(0.0, 0.0, 0.0), gravity=(0.0, -9.81, 0.0)):
        self._mask = mask
        nz, ny, nx = mask.shape
        self._st = SimpleNamespace(nx=nx, ny=ny, nz=nz, dx=dx, origin=SimpleNamespace(x=origin[0], y=origin[1],
                                                                                        z=origin[2]))
        self.fluid = sc.FluidParams(gravity=gravity)

    def stats(self):
        return self._st

    def cavity_mask(self):
        return self._mask.reshape(-1).astype(np.uint8)


def test_preseed_fills_deepest_cells_first():
    mask = np.zeros((4, 5, 6), dtype=bool)  # (z, y, x)
    mask[1:3, 1:4, 1:5] = True
    s = _FakeSolver(mask)
    pos, vel = preseed_pool(s, target=8 * 8 + 3)
    assert pos.shape == (67, 3) and not vel.any()
    cells = np.floor(pos / 1e-3).astype(int)  # jitter stays inside the cell
    # the lowest cavity layer (y = 1) holds 4 x 2 cells = 64 particles; the rest go one layer up
    assert np.all(cells[:64, 1] == 1) and np.all(cells[64:, 1] == 2)
    centre = (cells[0] + 0.5) * 1e-3
    assert np.array_equal(pos[0], centre + hash_jitter(np.array([0], dtype=np.uint64))[0] * 1e-3)
    full, _ = preseed_pool(s, target=10 ** 6)
    assert len(full) == mask.sum() * 8
