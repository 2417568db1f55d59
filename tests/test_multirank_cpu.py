"""The N>1 path of bench.py on CPU: world size 2 with the gloo backend.

The Stokes-limit path has no exchange step, so N GPUs run N independent
replicas; the only collective is the max-over-ranks of the timings.  These
tests run the same helper functions bench.py uses, in two processes.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    # rank r reports times 10 + r and 0.5 * (r + 1)
    out = bench.aggregate([10.0 + rank, 0.5 * (rank + 1)], dist, device="cpu")
    seed = bench.replica_seed(rank)
    seeds = [None] * world
    dist.all_gather_object(seeds, seed)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, out, seeds))


def test_two_ranks_take_the_max_and_distinct_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, out, seeds in res:
        assert out == [11.0, 1.0]
        assert len(set(seeds)) == 2  # every rank simulates its own replica


def test_single_process_aggregate_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.aggregate([3.0, 4.5]) == [3.0, 4.5]
