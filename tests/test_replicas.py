"""The N > 1 path (replicas, one process per GPU) on CPU: two gloo ranks, the same barrier /
max-over-ranks / throughput calls bench.py makes around its timed regions."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from rpp_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, ms, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    assert replicas.env() == (world, rank, rank)
    assert replicas.init("gloo", timeout_s=30) == world
    replicas.barrier()
    slowest = replicas.max_over_ranks(ms[rank])
    value = replicas.job_throughput(1000.0, slowest, world)
    replicas.barrier()
    replicas.finish()
    out.put((rank, slowest, value))


@pytest.mark.parametrize("world", [2])
def test_two_ranks_take_the_slowest_time(world):
    ms = [3.0, 5.0]   # rank 1 is the slow one
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, ms, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(out.get(timeout=10) for _ in range(world))
    for rank, slowest, value in got:
        assert slowest == 5.0                        # every rank sees the job's time
        assert value == pytest.approx(2 * 1000.0 / 5e-3)   # all ranks' units over the slowest time


def test_one_rank_without_a_launcher(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert replicas.env() == (1, 0, 0)
    assert replicas.init("gloo") == 1
    assert replicas.max_over_ranks(4.5) == 4.5
    assert replicas.job_throughput(10.0, 2.0, 1) == pytest.approx(5000.0)
