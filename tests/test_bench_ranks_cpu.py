"""bench.py's multi-rank reduction on CPU: two gloo ranks with different times
agree on the slowest rank's time, and the whole-job rate counts both ranks'
work over that time (weak scaling: one system per rank)."""
import os
import socket
import sys
from datetime import timedelta

import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def _rank(rank, world, port, q):
    sys.path.insert(0, REPO)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    mine = [1.5, 2.5][rank]
    t = bench.max_over_ranks(dist, mine, device="cpu")
    q.put((rank, t, bench.job_rate(1000, world, t)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[1] for g in got] == [2.5, 2.5]
    assert [g[2] for g in got] == [800.0, 800.0]


def test_single_process_is_unchanged():
    sys.path.insert(0, REPO)
    import bench
    assert bench.max_over_ranks(None, 3.25) == 3.25
    assert bench.job_rate(1048576, 1, 2.0) == 524288.0
