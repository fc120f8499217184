"""The multi-GPU path of bench.py is replicas only: each rank solves its own
copy of the workload and the job time is the slowest rank's. Checked with
two gloo ranks on the CPU (no GPU, no data-path collective)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, REPO)
    import datetime

    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    t = bench.max_over_ranks(1.0 + rank, dist)
    out[rank] = (t, bench.replica_throughput(world, 100, 3, t))
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_take_the_slowest_rank():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        for r in range(world):
            t, v = out[r]
            assert t == pytest.approx(2.0)
            assert v == pytest.approx(world * 100 * 3 / 2.0)
