"""The FP64 oracle, pinned against the reference's own CPU kernels (CPU only).

The reference ships no golden vectors; tests/golden/make_golden.py records
outputs of its CPU code (src/cpu_kernels/cpu_kernels.cpp, compiled
unmodified) and these tests check the oracle's restatement against them.
The reference computes in FP32 with a one-pass variance and its CPU kernel
uses the exclusion |i-1-j| < m (cpu_kernels.cpp:57), so comparisons use that
rule where flags are compared and skip windows within FP32 noise of r.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from paddi_b200 import datagen

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return json.load(open(os.path.join(G, name)))


def test_direct_and_recurrence_profiles_agree():
    x, _ = datagen.pd3_series(n=3000, seed=2, n_anom=3, anom_len=60)
    for m in (8, 40, 130):
        nn0, i0 = O.nn_profile(x, m, method=0)
        nn1, i1 = O.nn_profile(x, m, method=1)
        np.testing.assert_allclose(nn1, nn0, rtol=1e-10, atol=1e-9)
        assert np.mean(i0 == i1) > 0.999


def test_single_window_nn_matches_profile():
    x, _ = datagen.pd3_series(n=2000, seed=3, n_anom=2, anom_len=50)
    m = 33
    nn, idx = O.nn_profile(x, m)
    for i in (0, 17, 999, len(nn) - 1):
        d, j = O.window_nn(x, m, i)
        assert d == pytest.approx(nn[i], rel=1e-12)
        assert j == idx[i]


def test_statistics_vs_reference_cpu():
    f = np.load(os.path.join(G, "ref_stats.npz"))
    x = f["x"]
    for m in (8, 32, 100):
        mu, sd, flat = O.window_stats(x, m)
        np.testing.assert_allclose(f[f"mean_{m}"], mu, rtol=1e-5, atol=1e-4)
        # the reference's one-pass FP32 variance loses digits: std to 1e-2
        np.testing.assert_allclose(f[f"std_{m}"], sd, rtol=1e-2, atol=1e-3)
        assert not flat.any()


def test_candidate_flags_and_distances_vs_reference_cpu():
    meta = _load("ref_attempts.json")
    f = np.load(os.path.join(G, "ref_attempts.npz"))
    compared = 0
    for e in meta:
        x = f[f"x_{e['series']}"]
        m = e["m"]
        r2 = np.float32(e["r"]) * np.float32(e["r"])
        # the CPU kernel's exclusion rule: j admissible iff |i-1-j| >= m
        nn, _ = O.nn_profile(x, m, right_gap=m - 1, left_gap=m + 1)
        cand = f[f"cand_{e['key']}"].astype(bool)
        nnd = f[f"nnd_{e['key']}"]
        # survives iff every admissible d > r^2 (it prunes at d <= r, :62-70)
        want = nn > r2
        # outside the FP32 noise of the reference's formula, which errs in rho
        # (about 5e-4 at m = 16), i.e. by 2m * 5e-4 in distance units
        clear = np.abs(nn - r2) > 2 * m * 5e-4
        assert clear.mean() > 0.98
        np.testing.assert_array_equal(cand[clear], want[clear])
        s = cand & clear
        # the reference's raw-dot-product FP32 formula errs in rho, i.e. on the
        # scale of 2m in distance units
        np.testing.assert_allclose(nnd[s], nn[s], rtol=0, atol=2 * m * 2e-3)
        # attempt record: count of survivors and the top-1
        assert abs(e["n_cand"] - int(want.sum())) <= int((~clear).sum())
        if e["found"]:
            assert e["top_ind"] == int(np.argmax(np.where(want, nn, -np.inf)))
            assert e["top_dist"] == pytest.approx(nn[e["top_ind"]], rel=2e-3)
        compared += int(clear.sum())
    assert compared > 10000


def _series_b():
    rng = np.random.default_rng(12)
    x = datagen.random_walk_sine(2500, rng)
    datagen.plant_anomalies(x, [700, 1600], [48, 60], ["noise", "reverse"], rng)
    return x.astype(np.float32)


def test_palmad_schedule_vs_reference_cpu():
    ref = _load("ref_palmad.json")
    x = _series_b()
    disc, log = O.palmad(x, ref["minL"], ref["maxL"])
    assert [d[0] for d in disc] == [d[0] for d in ref["discords"]]
    for (_, a), (_, b) in zip(disc, ref["discords"]):
        assert a == pytest.approx(b, rel=1e-3)
    assert len(log) == len(ref["attempts"])
    for a, b in zip(log, ref["attempts"]):
        assert a["m"] == b["m"]
        assert a["found"] == b["found"]
        assert a["r2"] == pytest.approx(b["r2"], rel=1e-3)
        # counts differ only by the CPU kernel's shifted exclusion window
        assert abs(a["n_cand"] - b["n_cand"]) <= max(2, 0.002 * b["n_cand"])


def test_oracle_palmad_regression_fixture():
    want = _load("oracle_palmad.json")
    disc, log = O.palmad(_series_b(), want["minL"], want["maxL"])
    assert [list(d) for d in disc] == [list(d) for d in want["discords"]]
    assert log == want["attempts"]


def test_flat_window_policy():
    x = np.cumsum(np.random.default_rng(4).standard_normal(600)).astype(np.float32)
    x[100:160] = x[100]
    m = 20
    mu, sd, flat = O.window_stats(x, m)
    assert flat[100:141].all() and not flat[99] and not flat[141]
    assert (sd[flat] == 0).all()
    # flat vs non-flat: d = 2m; flat vs flat (admissible): d = 0
    assert O.pair_dist(x, m, 100, 300) == pytest.approx(2 * m)
    assert O.pair_dist(x, m, 100, 100 + m - 1) == 0.0


def test_select_semantics():
    nn = np.array([5.0, 9.0, 9.0, 3.0, 12.0, 12.0, 1.0])
    att, sel = O.select(nn, m=3, r2=4.0, top_k=3)
    assert (att["n_cand"], att["n_disc"]) == (5, 5)
    # first maximum wins (index 4; 3 and 5 overlap it: |i-j| < m-1), then 1
    # (first of the tied 9s; 0 and 2 overlap it); 6 is below r
    assert [s[0] for s in sel] == [4, 1]
    att, sel = O.select(nn, m=3, r2=9.0, top_k=1)
    assert (att["n_cand"], att["n_disc"]) == (4, 2)  # nn >= r2 vs nn > r2
