"""The multi-GPU bench path (scene replicas, one per rank; no collective on
the data path) on the CPU: two gloo ranks reduce their timings and counts
the way bench.py does — max of device and wall time over ranks, sum of the
particle-substeps — so whole-job throughput is the units of all ranks over
the slowest rank's time."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dev_ms = [120.0, 150.0][rank]
        wall = [0.20, 0.18][rank]
        ps = [1_000_000, 3_000_000][rank]
        out[rank] = bench.reduce_over_ranks(dev_ms, wall, ps, "cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_reduction_matches_bench_contract():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0] == res[1] == (150.0, 0.20, 4_000_000)
    dev_ms, wall, ps = res[0]
    assert abs(ps / (dev_ms / 1e3) - 4_000_000 / 0.150) < 1e-6


def test_substep_bytes_contract():
    import bench
    # one substep: 1000 particles, 10x10x10 cells, 20^3 SDF nodes, 500 fluid cells x 10 iterations
    b = bench.substep_bytes(1000, 1, 1000, 8000, 5000)
    assert b == 112 * 1000 + 92 * 1000 + 4 * 8000 + 83 * 5000
    assert bench.substep_bytes(2000, 2, 1000, 8000, 10000) == 2 * b
