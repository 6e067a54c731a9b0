"""Multi-replica timing plumbing of bench.py on two gloo ranks (CPU)."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    local_ms = 100.0 * (rank + 1)  # rank 1 is the slow one
    value, step = bench.replica_value(world, 1e12, local_ms)
    bench.barrier(world)
    q.put((rank, value, step))
    dist.destroy_process_group()


def test_two_gloo_replicas_report_the_max_step_time():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for _, value, step in res:
        assert step == pytest.approx(200.0)
        assert value == pytest.approx(2 * 1e12 / 0.2)
