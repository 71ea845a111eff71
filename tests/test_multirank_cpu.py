"""The N > 1 path of bench.py on CPU ranks (gloo, world size 2): replicas
reduce their times to the slowest rank's and aggregate the whole job's units;
the reference arm runs on rank 0 only."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        my_ms = 100.0 + 50.0 * rank                    # rank 1 is the slow one
        m = bench.max_over_ranks(my_ms, world, device="cpu")
        v = bench.replica_value(world, steps=10, units_per_step=1e6, max_ms=m)
        assert bench.dist_setup() == (world, rank, rank)
        q.put((rank, m, v))
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert [r[1] for r in res] == [150.0, 150.0]
    # 2 replicas x 10 steps x 1e6 units in 150 ms
    assert res[0][2] == pytest.approx(2 * 10 * 1e6 / 0.150)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class A:
        config, steps, warmup = 1, 1, 3

    assert bench.run_reference(A()) == 0   # returns at once, no work, no output
