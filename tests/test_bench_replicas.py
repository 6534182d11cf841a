"""The replica path of bench.py (N > 1 under torchrun): every rank renders an
independent replica, the job's step time is the slowest rank's and its rate
is N times that. Exercised with world_size-2 gloo process groups on CPU."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, ms, rates, out):
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    try:
        ms_max, value = bench.replica_throughput(ms[rank], world, dist, torch.device("cpu"))
        rate = bench.replica_rate(rates[rank], world, dist, torch.device("cpu"))
        out.put((rank, ms_max, value, rate))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world, port = 2, _free_port()
    ms, rates = [0.8, 1.25], [300.0, 240.0]
    procs = [ctx.Process(target=_worker, args=(r, world, port, ms, rates, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=100) for _ in range(world)]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    for rank, ms_max, value, rate in res:
        assert ms_max == pytest.approx(1.25)
        assert value == pytest.approx(2 * 1000.0 / 1.25)
        assert rate == pytest.approx(2 * 240.0)


def test_single_rank_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    ms_max, value = bench.replica_throughput(0.5, 1, None, torch.device("cpu"))
    assert ms_max == 0.5 and value == pytest.approx(2000.0)
    assert bench.replica_rate(10.0, 1, None, torch.device("cpu")) == 10.0
