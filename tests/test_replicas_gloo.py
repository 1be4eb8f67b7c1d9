"""Multi-process replica aggregation of bench.py (world size 2, gloo on CPU): the step time is the
max over ranks and the value the sum of the ranks' DOF over that time."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        d = bench._TorchDist(torch, dist, device="cpu")
        ms = [10.0, 12.5][rank]              # per-rank device time of the K timed steps
        dof = [1.0e6, 2.0e6][rank]
        ms_step, value = bench.replica_throughput(d, ms, 5, dof)
        d.barrier()
        out[rank] = (ms_step, value)
    finally:
        dist.destroy_process_group()


def test_replica_throughput_two_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        ms_step, value = out[r]
        assert ms_step == pytest.approx(12.5 / 5)
        assert value == pytest.approx(3.0e6 / (2.5e-3))
