"""The N>1 bench path on CPU ranks (gloo, world size 2): every rank runs a
replica; the job rate uses the slowest rank's time."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    local = 1.0 + rank          # rank 1 is the slow replica
    t = bench.max_over_ranks(local, dist, "cpu")
    rate = bench.aggregate_rate(cells=1000, stages=3, seconds_max=t, world=world)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, t, rate))


def test_two_rank_max_and_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, rate in res:
        assert t == 2.0
        assert abs(rate - 2 * 1000 * 3 / 2.0 / 1e9) < 1e-18
