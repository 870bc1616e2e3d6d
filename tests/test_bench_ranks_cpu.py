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


def _lpt_rank(rank, world, port, q):
    sys.path.insert(0, REPO)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))

    import numpy as np
    rng = np.random.default_rng(2024)
    sizes = [int(round(float(np.exp(rng.uniform(np.log(4096), np.log(65536)))))) for _ in range(64)]
    mine = bench.lpt_split([float(n) for n in sizes], world)[rank]
    views = [None] * world
    dist.all_gather_object(views, mine)
    q.put((rank, mine, views, sizes))
    dist.barrier()
    dist.destroy_process_group()


def test_lpt_split_over_two_gloo_ranks():
    """Replica placement for bench.py --gpus N: each rank computes its share of
    the 64-replica batch from the same sizes, with no exchange; the shares are
    disjoint, cover every replica, and differ in total size by at most the
    largest replica (the longest-processing-time bound)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_lpt_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, m0, v0, sizes), (_, m1, v1, _) = got
    assert v0 == v1 == [m0, m1]
    assert sorted(m0 + m1) == list(range(64))
    loads = [sum(sizes[i] for i in m) for m in (m0, m1)]
    assert abs(loads[0] - loads[1]) <= max(sizes)


def test_lpt_split_single_rank_and_ties():
    sys.path.insert(0, REPO)
    import bench
    assert bench.lpt_split([3.0, 1.0, 2.0], 1) == [[0, 1, 2]]
    assert bench.lpt_split([5.0, 5.0, 5.0, 5.0], 2) == [[0, 2], [1, 3]]
    assert bench.lpt_split([], 3) == [[], [], []]


def test_reference_arm_prints_the_contract_line():
    """`bench.py --impl reference` (the reference's own attempt_monte_carlo_move
    from oracle/_ref, on the host cores) prints one JSON line with the GPU arm's
    metric, unit and config, its real timed steps, and e2e equal to value."""
    import json
    import subprocess

    import pytest
    if not os.path.exists(os.path.join(REPO, "oracle", "_ref", "libmcref_omp.so")):
        pytest.skip("oracle/_ref not built (the reference source was not available at build time)")
    sys.path.insert(0, REPO)
    import bench
    out = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "3",
                          "--warmup", "1", "--cpu-seconds", "2"], capture_output=True, text=True, timeout=600,
                         cwd=REPO)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["config"] == bench.WORKLOAD and d["steps"] == 3 and d["warmup"] == 1
    assert d["value"] > 0 and d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert d["ms_per_step"] > 0 and d["higher_is_better"] is True
