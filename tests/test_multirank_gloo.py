"""Multi-rank bookkeeping of bench.py on CPU (gloo, world size 2): the job's
time is the slowest rank's, and the throughput counts every rank's units."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    times = [10.0 + rank, 3.0 * (2 - rank), 1.5]
    mx = bench.max_over_ranks(times, world)
    rate = bench.job_rate(64 * 16 * 10, world, mx[0])
    q.put((rank, mx, rate))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_rate_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, rate in out:
        assert mx == [11.0, 6.0, 1.5]
        assert rate == pytest.approx(64 * 16 * 10 * 2 / 0.011)
