"""The multi-process side of bench.py on the CPU: two gloo ranks hand their
timed and end-to-end figures to over_ranks, which must return the slowest
rank's times and the sum of all ranks' rays on every rank (the figures a
replicated --gpus N run reports)."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, results):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        results[rank] = bench.over_ranks(dist, "cpu", 10.0 * rank + 5.0, 100 + rank, 7.0 + rank, 50)
    finally:
        dist.destroy_process_group()


def test_over_ranks_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as manager:
        results = manager.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, results)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        got = dict(results)
    for rank in range(2):
        assert got[rank] == (15.0, 201, 8.0, 100)


def test_over_ranks_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.over_ranks(None, "cpu", 12.5, 7, 3.0, 9) == (12.5, 7, 3.0, 9)
