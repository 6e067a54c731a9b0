"""The sharded PALMAD / PD3 driver on two gloo ranks (CPU).

Each rank runs the exact oracle backend (tests/shard_oracle.py) on its rows
and columns; the exchanges are real torch.distributed collectives.  The
sharded run must give the single-process oracle's discords and attempt
counts, and every merged candidate value must equal the whole range's (the
backend asserts it).
"""
import os
import socket

import numpy as np
import pytest

from paddi_b200 import sharded


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _series():
    from paddi_b200 import datagen
    x, _ = datagen.palmad_series(n=2600, seed=9, n_anom=3, min_len=30, max_len=60)
    return x


def _rank(rank, world, port, q, what):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        from tests.shard_oracle import OracleBackend
        be = OracleBackend(_series(), seed=rank)
        comm = sharded.TorchComm(device="cpu")
        if what == "palmad":
            disc, logs = sharded.palmad_sharded(be, comm, 40, 45)
            q.put((rank, [(d.ind, d.dist) for d in disc],
                   [(e["n_cand"], e["n_disc"]) for e in logs]))
        else:
            disc, logs = sharded.pd3_sharded(be, comm, 48, top_k=3)
            q.put((rank, [(d.ind, d.dist) for d in disc],
                   [(e["n_cand"], e["n_disc"]) for e in logs]))
    finally:
        dist.destroy_process_group()


def _run(what, world=2):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q, what)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    return sorted(q.get(timeout=10) for _ in range(world))


def test_shard_ranges_cover_the_windows_on_the_tile_grid():
    for N, world in [(100000, 2), (2_096_641, 8), (5000, 3), (1000, 4)]:
        rows, cols = sharded.shard_ranges(N, world)
        assert rows[0][0] == 0 and rows[-1][1] == N
        assert all(a[1] == b[0] for a, b in zip(rows, rows[1:]))
        assert cols[0][0] == 0 and cols[-1][1] == N
        assert all(a[1] == b[0] for a, b in zip(cols, cols[1:]))
        assert all(lo % sharded.TILE == 0 for lo, _ in cols)


def test_two_gloo_ranks_give_the_single_process_palmad():
    from oracle import oracle as O
    res = _run("palmad")
    want, watt = O.palmad(_series(), 40, 45)
    for _, disc, counts in res:
        assert [d[0] for d in disc] == [w[0] for w in want]
        for d, w in zip(disc, want):
            assert abs(d[1] - w[1]) <= 1e-6 * abs(w[1])
        assert counts == [(a["n_cand"], a["n_disc"]) for a in watt]


def test_two_gloo_ranks_give_the_single_process_pd3_topk():
    from oracle import oracle as O
    res = _run("pd3")
    want, watt = O.pd3(_series(), 48, top_k=3)
    for _, disc, counts in res:
        assert [d[0] for d in disc] == [w[0] for w in want]
        assert counts == [(a["n_cand"], a["n_disc"]) for a in watt]


def test_three_thread_ranks_give_the_single_process_palmad():
    """The same driver with ranks as threads of one process (ThreadComm): three
    uneven shards, the exact CPU backend per rank."""
    import threading

    from oracle import oracle as O
    from tests.shard_oracle import OracleBackend
    x = _series()
    comms = sharded.ThreadComm.group(3)
    res = [None] * 3

    def run(rank):
        disc, logs = sharded.palmad_sharded(OracleBackend(x, seed=rank), comms[rank], 40, 45)
        res[rank] = ([(d.ind, d.dist) for d in disc], [(e["n_cand"], e["n_disc"]) for e in logs])

    ts = [threading.Thread(target=run, args=(r,)) for r in range(3)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(300)
    want, watt = O.palmad(x, 40, 45)
    for disc, counts in res:
        assert [d[0] for d in disc] == [w[0] for w in want]
        for d, w in zip(disc, want):
            assert abs(d[1] - w[1]) <= 1e-6 * abs(w[1])
        assert counts == [(a["n_cand"], a["n_disc"]) for a in watt]
