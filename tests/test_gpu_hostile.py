"""GPU parity on series built to stress the distance kernels' rounding.

A refine kernel's error for the pair (candidate, window j) grows with the
ratio |mean_j - tile level| / std_j; phase 1's with the norms of the windows
its walk passes.  These series push those ratios up: stretches whose values
vary by 1e-5 of the walk's range, a 1e4 offset with unit local variance,
integer-quantised values with many ties and flat runs, an ECG-like series
with a flat noisy baseline.  For every refine kernel (FP32, split-FP16,
split-BF16) the library must give the oracle's results exactly: the same
candidate and discord counts at thresholds spread over the nn distribution,
the same top-k windows, and FP64-exact distances (tolerance 1e-5 relative,
the parity tolerance of the other GPU tests).
"""
import numpy as np
import pytest

import paddi_b200 as P
from oracle import oracle as O
from paddi_b200 import datagen

pytestmark = pytest.mark.gpu

KINDS = ["near_flat", "offset", "quantised", "ecg_flat"]
DISTS = {"fp32": P.DIST_FP32, "fp16": P.DIST_SPLIT_FP16, "bf16": P.DIST_SPLIT_BF16}
DIST_RTOL = 1e-5


def _close(a, b):
    return abs(a - b) <= DIST_RTOL * max(abs(a), abs(b), 1e-30)


_SERIES = {}


def _series(kind):
    if kind not in _SERIES:
        _SERIES[kind] = datagen.hostile_series(kind, n=1 << 14, seed=7)[0]
    return _SERIES[kind]


@pytest.fixture(scope="module", params=sorted(DISTS))
def ctx(request):
    c = P.Context(device=0, distance_kernel=DISTS[request.param])
    yield c
    c.close()


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("m", [64, 150])
def test_attempt_counts_and_topk_on_hostile_series(ctx, kind, m):
    x = _series(kind)
    nn, _ = O.nn_profile(x, m)
    finite = nn[np.isfinite(nn)]
    for q in (0.5, 0.99, 0.999):
        r = float(np.sqrt(np.float32(np.quantile(finite, q))))
        r2f = np.float32(r) * np.float32(r)
        att, sel = O.select(nn, m, float(r2f), top_k=3)
        got, log = ctx.pd3(x, m, top_k=3, r=r)
        assert (log[0]["n_cand"], log[0]["n_disc"]) == (att["n_cand"], att["n_disc"]), (kind, q)
        assert [d.ind for d in got] == [s[0] for s in sel], (kind, q, got, sel)
        for d, s in zip(got, sel):
            assert _close(d.dist, s[1]), (kind, q, d, s)


@pytest.mark.parametrize("kind", KINDS)
def test_palmad_on_hostile_series(ctx, kind):
    x = _series(kind)
    minL, maxL = 96, 101
    want, watt = O.palmad(x, minL, maxL)
    got, log = ctx.palmad(x, minL, maxL)
    assert [d.ind for d in got] == [w[0] for w in want]
    for d, w in zip(got, want):
        assert _close(d.dist, w[1]), (d, w)
    assert [(e["n_cand"], e["n_disc"]) for e in log] == \
        [(a["n_cand"], a["n_disc"]) for a in watt]


def test_hostile_series_reach_the_fragile_pass():
    # the near-flat stretches have windows whose split-16-bit rounding bound is
    # above the guard band: the refine must hand them to the FP64 pass
    x = _series("near_flat")
    with P.Context(device=0, distance_kernel=P.DIST_SPLIT_FP16) as c:
        _, log = c.pd3(x, 150, top_k=1)
    assert max(e["n_fragile"] for e in log) > 0
