"""The bench's multi-GPU plumbing (replicas, one process per GPU, no data-path
collective: one problem does not shard) on world_size 2 over gloo on the CPU:
the job's time is the slowest replica's, its ms per solve counts every
replica's solves."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        totals = [30.0, 50.0]  # ms of 10 steps on each replica
        out[rank] = (bench.max_over_ranks(totals[rank], world), bench.replica_value(totals[rank], 10, world))
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_replicas_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    for r in range(2):
        mx, v = res[r]
        assert mx == 50.0
        assert v == pytest.approx(50.0 / 20)
