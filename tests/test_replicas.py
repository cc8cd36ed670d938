"""Multi-GPU mode of the benchmark: independent replicas (one design and its
own stimulus streams per rank), timed as the max over ranks, whole-job value
= all ranks' units over that time.  Runs the rank logic as two gloo
processes on the CPU."""
import os
import socket
import sys

import pytest
import torch
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, HERE)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        # rank r takes (r + 1) * 10 ms of device time, (r + 1) * 12 ms end to end
        v, e, dev_ms, e2e_ms = bench.replica_throughput(1000, 10.0 * (rank + 1), 12.0 * (rank + 1),
                                                        world, device="cpu")
        out[rank] = (v, e, dev_ms, e2e_ms)
    finally:
        dist.destroy_process_group()


def test_replica_throughput_is_max_over_ranks():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    assert sorted(out.keys()) == [0, 1]
    for r in range(world):
        v, e, dev_ms, e2e_ms = out[r]
        assert dev_ms == pytest.approx(20.0) and e2e_ms == pytest.approx(24.0)
        assert v == pytest.approx(world * 1000 / 0.020)
        assert e == pytest.approx(world * 1000 / 0.024)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, HERE)
    import bench
    v, e, dev_ms, e2e_ms = bench.replica_throughput(500, 5.0, 10.0, 1)
    assert (v, e, dev_ms, e2e_ms) == (pytest.approx(100000.0), pytest.approx(50000.0), 5.0, 10.0)
