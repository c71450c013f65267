"""bench.py --gpus N runs N independent replicas of the solve (one per rank,
no collective on the data path): the job's time is the slowest rank's and
its throughput all ranks' solves over that time. The reduction and the
arithmetic, on two CPU ranks over gloo."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}",
                            rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = 100.0 * (rank + 1)  # rank 1 is the slower replica
        worst = bench.max_over_ranks(world, ms)
        out.put((rank, worst, bench.replicas_value(world, 10, worst)))
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q))
             for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[1] for g in got] == [200.0, 200.0]
    # two replicas of 10 solves each, the slower in 0.2 s: 100 solves/s
    assert all(abs(g[2] - 100.0) < 1e-9 for g in got)
