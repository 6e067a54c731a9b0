"""Parity at the full sizes of the benchmarked configurations.

* The headline PALMAD run: n = 2^21 (``datagen.palmad_series(seed=1)``),
  lengths 64..512, top-1, learned r and the split-FP16 refine, exactly as
  bench.py times it.  At the lengths of ``tests/golden/c2_top1.json`` the
  reported window and distance must equal the top-1 of the full FP64 nn
  profile (every window against every admissible window, computed offline by
  ``tests/golden/make_c2_fixture.py``); at every one of the 449 lengths the
  reported distance must equal the FP64 nn of the reported window.
* PD3 at the fixed-length configuration: n = 131072, m = 128, segment
  length 4096, top-4, the halving r-schedule from 2 sqrt(m), against the
  oracle's full FP64 profile: the same windows, distances and attempts.

Distances are FP64 values rounded to float on both sides; the tolerance
written here (1e-6 relative) only absorbs the last-bit rounding differences
of two FP64 evaluation orders.  The north-star bar is 1e-4.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import paddi_b200 as P
from oracle import oracle as O
from paddi_b200 import datagen

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
DIST_RTOL = 1e-6


def _close(a, b, rtol=DIST_RTOL):
    return abs(a - b) <= rtol * max(abs(a), abs(b), 1e-30)


@pytest.fixture(scope="module")
def headline():
    fx = json.load(open(os.path.join(HERE, "golden", "c2_top1.json")))
    x, _ = datagen.palmad_series(n=1 << 21, seed=1)
    assert hashlib.sha256(np.ascontiguousarray(x, np.float32).tobytes()).hexdigest() == \
        fx["sha256"], "the series generator changed: regenerate the fixture"
    with P.Context(device=0, distance_kernel=P.DIST_AUTO, r_policy=P.R_LEARNED) as ctx:
        disc, log = ctx.palmad(x, 64, 512)
    return x, fx, disc, log


def test_headline_top1_equals_the_full_fp64_profile(headline):
    x, fx, disc, _ = headline
    assert len(fx["lengths"]) >= 4
    for m, e in sorted(fx["lengths"].items(), key=lambda kv: int(kv[0])):
        d = disc[int(m) - 64]
        assert d.ind == e["ind"], (m, d, e)
        assert _close(d.dist, e["dist"]), (m, d, e)


def test_headline_every_distance_is_the_fp64_nn_of_its_window(headline):
    x, _, disc, log = headline
    w = [d.ind for d in disc]
    assert min(w) >= 0
    exact = O.lengths_nn(x, 64, 512, w)
    bad = [(64 + q, disc[q], exact[q]) for q in range(len(w))
           if not _close(disc[q].dist, float(np.float32(exact[q])))]
    assert not bad, bad[:5]
    # the attempts found their discords at every length
    assert {e["m"] for e in log if e["found"]} == set(range(64, 513))


def test_fixed_length_config_matches_the_oracle():
    x, _ = datagen.pd3_series(n=131072, seed=0)
    m, k = 128, 4
    with P.Context(device=0) as ctx:
        got, log = ctx.pd3(x, m, top_k=k, segment_len=4096)
    want, wlog = O.pd3(x, m, top_k=k, fast=True)
    assert [d.ind for d in got] == [w[0] for w in want]
    for d, w in zip(got, want):
        assert _close(d.dist, w[1]), (d, w)
    assert [(e["r2"], e["n_cand"], e["n_disc"]) for e in log] == \
        [(np.float32(a["r2"]), a["n_cand"], a["n_disc"]) for a in wlog]


def test_segment_lengths_beyond_the_supported_range_are_refused():
    x, _ = datagen.pd3_series(n=16384, seed=0)
    with P.Context(device=0) as ctx:
        with pytest.raises(P.PaddiError) as e:
            ctx.pd3(x, 128, top_k=1, segment_len=8192)
        assert e.value.status == P.PADDI_ERR_UNSUPPORTED
    with pytest.raises(P.PaddiError) as e:
        P.Context(device=0, segment_len=32)
    assert e.value.status == P.PADDI_ERR_UNSUPPORTED


def test_large_run_reports_exact_distances_at_sampled_lengths():
    """Config C5 at full size (ECG-like n = 2^27, lengths 128..384, learned r):
    every length finds its discord, and at 8 lengths spread over the range the
    reported distance is the FP64 nn of the reported window (a full FP64
    profile is out of reach at this size: one length is ~1e16 pair terms)."""
    x, _ = datagen.ecg_series(n=1 << 27, seed=5)
    minL, maxL = 128, 384
    with P.Context(device=0, r_policy=P.R_LEARNED) as ctx:
        disc, log = ctx.palmad(x, minL, maxL)
    assert {e["m"] for e in log if e["found"]} == set(range(minL, maxL + 1))
    for m in (128, 129, 160, 200, 256, 300, 350, 384):
        d = disc[m - minL]
        nn, _ = O.windows_nn(x, m, [d.ind])
        assert _close(d.dist, float(np.float32(nn[0]))), (m, d, nn[0])
