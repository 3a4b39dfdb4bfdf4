"""Multi-GPU runs are independent replicas (the step does not shard): the job's
throughput is every rank's steps over the slowest rank's time.  The rank logic of
bench.py runs here as world_size 2 over gloo on the CPU."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        # rank r timed 100 steps in 10 (r + 1) ms
        q.put((rank, bench.replica_throughput(10.0 * (rank + 1), 100, world, "cpu")))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replica_throughput_two_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(2):
        t_max, value = out[r]
        assert t_max == pytest.approx(20.0)
        assert value == pytest.approx(2 * 100 / 0.020)


def test_replica_throughput_one_rank():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.replica_throughput(5.0, 10, 1, "cpu") == (5.0, 2000.0)
