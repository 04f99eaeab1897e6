"""Replica (multi-GPU) bookkeeping of bench.py on CPU with gloo, world size 2.

The path runs one independent replica per GPU (no data-path collective); the
job's time is the slowest rank's and its throughput counts every replica.
"""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import datetime
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    local_ms = 10.0 + 5.0 * rank                  # rank 1 is the slower replica
    mx = bench.max_over_ranks(local_ms, dist, "cpu")
    val = bench.job_throughput(world, 1000, 20, mx)
    q.put((rank, mx, val))
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_take_the_slowest_rank():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, val in res:
        assert mx == 15.0
        assert val == pytest.approx(2 * 1000 * 20 / 15e-3 / 1e9)


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    assert bench.job_throughput(1, 4186116, 200, 10.0) == pytest.approx(4186116 * 200 / 0.01 / 1e9)
