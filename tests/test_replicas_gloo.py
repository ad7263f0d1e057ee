"""Multi-process (world size 2, gloo on CPU) check of the replica timing in bench.py:
each rank proves its own instances, the job time is the maximum over ranks."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    bench.barrier(world)
    elapsed = bench.dist_max(10.0 * (rank + 1), world)
    seed = bench.replica_input_seed(world, rank)
    q.put((rank, elapsed, seed))
    dist.destroy_process_group()


def test_replica_max_over_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(world))
    assert [r[1] for r in res] == [20.0, 20.0]          # every rank sees the slowest rank's time
    assert [r[2] for r in res] == [0, 1]                # distinct input streams per replica
