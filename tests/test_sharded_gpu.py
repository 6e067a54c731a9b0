"""The sharded driver over libpaddi's shard entry points on one GPU.

Two ranks run as threads of this process, each with its own context and
stream on the same GPU; their exchanges are host-side (ThreadComm), so no
kernel waits for another.  The sharded PALMAD and PD3 runs must equal the
single-context runs and the FP64 oracle: same windows, same attempt counts,
distances within 1e-5 relative.
"""
import threading

import numpy as np
import pytest

import paddi_b200 as P
from oracle import oracle as O
from paddi_b200 import datagen, sharded

pytestmark = pytest.mark.gpu


def _threads(world, fn):
    comms = sharded.ThreadComm.group(world)
    res, errs = [None] * world, []

    def run(r):
        try:
            with P.Context(device=0, distance_kernel=P.DIST_AUTO) as ctx:
                res[r] = fn(ctx, comms[r])
        except Exception as e:  # reported below
            errs.append(e)
            comms[r].s.barrier.abort()

    ts = [threading.Thread(target=run, args=(r,)) for r in range(world)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(600)
    assert not errs, errs
    return res


@pytest.mark.parametrize("world", [1, 2, 3])
def test_sharded_palmad_equals_the_single_gpu_run(world):
    x, _ = datagen.palmad_series(n=1 << 17, seed=3, n_anom=6, min_len=40, max_len=120)
    minL, maxL = 60, 64
    with P.Context(device=0) as ctx:
        want, wlog = ctx.palmad(x, minL, maxL)

    def fn(ctx, comm):
        be = sharded.GpuBackend(ctx, x, device=0)
        return sharded.palmad_sharded(be, comm, minL, maxL)

    for disc, logs in _threads(world, fn):
        assert [d.ind for d in disc] == [d.ind for d in want]
        assert [d.dist for d in disc] == [d.dist for d in want]
        assert [(e["n_cand"], e["n_disc"]) for e in logs] == \
            [(e["n_cand"], e["n_disc"]) for e in wlog]


def test_sharded_pd3_topk_equals_the_oracle():
    x, _ = datagen.pd3_series(n=16384, seed=0, n_anom=4, anom_len=150)
    want, watt = O.pd3(x, 128, top_k=4)

    def fn(ctx, comm):
        return sharded.pd3_sharded(sharded.GpuBackend(ctx, x, device=0), comm, 128, top_k=4)

    for disc, logs in _threads(2, fn):
        assert [d.ind for d in disc] == [w[0] for w in want]
        for d, w in zip(disc, want):
            assert abs(d.dist - w[1]) <= 1e-5 * abs(w[1])
        assert [(e["n_cand"], e["n_disc"]) for e in logs] == \
            [(a["n_cand"], a["n_disc"]) for a in watt]


def test_shard_refine_rejects_columns_off_the_tile_grid():
    x, _ = datagen.pd3_series(n=16384, seed=0)
    with P.Context(device=0) as ctx:
        be = sharded.GpuBackend(ctx, x, device=0)
        alive = be.phase1(128, 100.0, 0, 1000)
        with pytest.raises(P.PaddiError) as e:
            be.refine(128, 100.0, alive, 100, 5000)
        assert e.value.status == P.PADDI_ERR_INVALID_ARG
