"""Failure detection without a GPU fault.

The reference exits the process on any CUDA error (src/common.h:6-16).  The
library returns a status instead and keeps the context usable.  These tests
make the failures happen on purpose, in forms that fault nothing:
  * a device allocation that fails on the host (a test hook makes the
    context's next allocation report cudaErrorMemoryAllocation);
  * a barrier wait of the tensor-core refine that runs out: the refine is
    told to withhold one pipeline stage (no copy or MMA is issued for it) and
    its wait limit is set to about 0.1 s.  The kernel records the timeout,
    waits (bounded) for what it did issue, frees its tensor memory and returns.
After each failure the same context must run a clean search that matches the
FP64 oracle.
"""
import numpy as np
import pytest

import paddi_b200 as P
from oracle import oracle as O
from paddi_b200 import datagen

pytestmark = pytest.mark.gpu


def _series():
    x, _ = datagen.palmad_series(n=1 << 13, seed=21, n_anom=4, min_len=32, max_len=96)
    return x


def _check_against_oracle(ctx, x, m, top_k=2):
    got, _ = ctx.pd3(x, m, top_k=top_k)
    want, _ = O.pd3(x, m, top_k=top_k)
    assert [d.ind for d in got] == [w[0] for w in want]
    for d, w in zip(got, want):
        assert abs(d.dist - w[1]) <= 1e-5 * abs(w[1])


def test_failed_allocation_returns_out_of_memory_and_the_context_recovers():
    x = _series()
    with P.Context(device=0) as ctx:
        ctx.debug_set(P.DEBUG_FAIL_ALLOC, 3)  # the third allocation of the next call
        with pytest.raises(P.PaddiError) as e:
            ctx.pd3(x, 64, top_k=2)
        assert e.value.status == P.PADDI_ERR_OUT_OF_MEMORY
        assert ctx.debug_get(P.DEBUG_FAIL_ALLOC) == 0  # consumed
        _check_against_oracle(ctx, x, 64)


@pytest.mark.parametrize("dist", [P.DIST_SPLIT_FP16, P.DIST_SPLIT_BF16])
def test_refine_wait_timeout_is_reported_once_and_the_context_recovers(dist):
    x = _series()
    m = 80
    nn, _ = O.nn_profile(x, m)
    r = float(np.sqrt(np.float32(np.quantile(nn, 0.99))))  # some candidates reach the refine
    with P.Context(device=0, distance_kernel=dist) as ctx:
        ctx.debug_set(P.DEBUG_WAIT_CYCLES, 200_000_000)  # ~0.1 s at 1.9 GHz
        ctx.debug_set(P.DEBUG_WITHHOLD_STAGE, 1)
        with pytest.raises(P.PaddiError) as e:
            ctx.pd3(x, m, top_k=1, r=r)
        assert e.value.status == P.PADDI_ERR_CUDA
        assert "timed out" in str(e.value)
        # the host returned at once: one selection pass, no redo of the refine
        assert ctx.debug_get(P.DEBUG_LAST_PASSES) == 1
        ctx.debug_set(P.DEBUG_WITHHOLD_STAGE, 0)
        ctx.debug_set(P.DEBUG_WAIT_CYCLES, 0)
        _check_against_oracle(ctx, x, m)


def test_debug_hooks_reject_unknown_keys():
    with P.Context(device=0) as ctx:
        with pytest.raises(P.PaddiError):
            ctx.debug_set(99, 1)
        with pytest.raises(P.PaddiError):
            ctx.debug_set(P.DEBUG_FAIL_ALLOC, -1)


def test_recheck_queue_grows_when_a_selection_overflows_it():
    """A selection that needs more exact values than the FP64 recheck queue
    holds must report the full count, grow the queue and redo the selection
    (a queue of one window overflows on the top-4 picks alone)."""
    x = _series()
    m = 64
    with P.Context(device=0) as ctx:
        ctx.reserve(len(x), m)
        ctx.debug_set(P.DEBUG_RECHECK_CAP, 1)
        got, log = ctx.pd3(x, m, top_k=4)
        assert ctx.debug_get(P.DEBUG_RECHECK_CAP) > 1
    want, wlog = O.pd3(x, m, top_k=4)
    assert [d.ind for d in got] == [w[0] for w in want]
    for d, w in zip(got, want):
        assert abs(d.dist - w[1]) <= 1e-5 * abs(w[1])
    assert [(e["n_cand"], e["n_disc"]) for e in log] == \
        [(a["n_cand"], a["n_disc"]) for a in wlog]
