"""GPU parity: libpaddi (through its C ABI) against the FP64 oracle.

Every case runs the CUDA library and the oracle on the same seeded input.
Bars: start indices, candidate / discord counts and attempt outcomes are
exact; reported squared distances agree within 1e-5 relative (they are FP64
values rounded to float on both sides, so in practice they are identical).
"""
import numpy as np
import pytest

from oracle import oracle as O
from paddi_b200 import datagen

P = pytest.importorskip("paddi_b200")

pytestmark = pytest.mark.gpu

DIST_RTOL = 1e-5


@pytest.fixture(scope="module")
def ctx():
    c = P.Context(distance_kernel=P.DIST_AUTO)
    yield c
    c.close()


@pytest.fixture(scope="module")
def ctx32():
    c = P.Context(distance_kernel=P.DIST_FP32)
    yield c
    c.close()


def _series(n, seed, kind="pd3"):
    if kind == "pd3":
        x, _ = datagen.pd3_series(n=n, seed=seed, n_anom=4, anom_len=min(150, n // 40))
    else:
        x, _ = datagen.palmad_series(n=n, seed=seed, n_anom=4, min_len=32, max_len=96)
    return x


def _close(a, b, rtol=DIST_RTOL):
    return abs(a - b) <= rtol * max(abs(a), abs(b), 1e-30)


# ------------------------------------------------------------------ statistics
@pytest.mark.parametrize("m", [16, 100, 257])
def test_statistics_match_oracle(ctx, m):
    import torch
    x = _series(6000, 3)
    mu, sd, _ = O.window_stats(x, m)
    dT = torch.from_numpy(x).cuda()
    N = len(x) - m + 1
    dm = torch.empty(N, dtype=torch.float32, device="cuda")
    ds = torch.empty(N, dtype=torch.float32, device="cuda")
    ctx.compute_statistics(dT.data_ptr(), dm.data_ptr(), ds.data_ptr(), len(x), m)
    torch.cuda.synchronize()
    np.testing.assert_allclose(dm.cpu().numpy(), mu, rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(ds.cpu().numpy(), sd, rtol=2e-6, atol=1e-7)


# ------------------------------------------------------------- single attempts
@pytest.mark.parametrize("n,m", [(4096, 32), (8192, 64), (8192, 128)])
@pytest.mark.parametrize("q", [0.5, 0.99, 0.9995, 1.01])
def test_pd3_attempt_counts_and_topk(ctx32, n, m, q):
    x = _series(n, 11 + m)
    nn, _ = O.nn_profile(x, m)
    r2 = float(np.float32(np.quantile(nn, q) if q < 1 else nn.max() * q))
    r = float(np.sqrt(np.float32(r2)))
    r2f = np.float32(r) * np.float32(r)
    att, sel = O.select(nn, m, float(r2f), top_k=3)
    got, log = ctx32.pd3(x, m, top_k=3, r=r)
    assert len(log) == 1
    assert log[0]["n_cand"] == att["n_cand"]
    assert log[0]["n_disc"] == att["n_disc"]
    assert [d.ind for d in got] == [s[0] for s in sel]
    for d, s in zip(got, sel):
        assert _close(d.dist, s[1])


def test_pd3_halving_topk4_matches_oracle(ctx):
    # the fixed-length workload (n=131072, m=128, k=4) at 1/8 scale
    x, _ = datagen.pd3_series(n=16384, seed=0, n_anom=4, anom_len=150)
    m = 128
    want, watt = O.pd3(x, m, top_k=4)
    got, log = ctx.pd3(x, m, top_k=4)
    assert [d.ind for d in got] == [w[0] for w in want]
    for d, w in zip(got, want):
        assert _close(d.dist, w[1])
    assert len(log) == len(watt)
    for a, b in zip(log, watt):
        assert a["r2"] == pytest.approx(b["r2"], rel=0, abs=0)
        assert (a["n_cand"], a["n_disc"]) == (b["n_cand"], b["n_disc"])


# ---------------------------------------------------------------------- PALMAD
@pytest.mark.parametrize("kind,n,minL,maxL", [("pd3", 8192, 32, 44), ("palmad", 8192, 40, 52)])
def test_palmad_matches_oracle(ctx, kind, n, minL, maxL):
    x = _series(n, 5, kind)
    want, watt = O.palmad(x, minL, maxL)
    got, log = ctx.palmad(x, minL, maxL)
    assert [d.ind for d in got] == [w[0] for w in want]
    for d, w in zip(got, want):
        assert _close(d.dist, w[1])
    assert len(log) == len(watt)
    for a, b in zip(log, watt):
        assert a["m"] == b["m"]
        assert a["r2"] == b["r2"]
        assert a["found"] == b["found"]
        assert (a["n_cand"], a["n_disc"]) == (b["n_cand"], b["n_disc"])


def test_range_discord_profile(ctx):
    """paddi_palmad_profiled: same discords as paddi_palmad; per length, the
    profile marks exactly the final attempt's candidates, holds the reported
    top-1 distance bit for bit at its window, and agrees with the oracle's
    FP64 nn profile within the refine's guard band elsewhere."""
    x = _series(8192, 5, "palmad")
    minL, maxL = 40, 46
    d, log, profs = ctx.palmad_profiled(x, minL, maxL)
    d2, _ = ctx.palmad(x, minL, maxL)
    assert [(q.ind, q.dist) for q in d] == [(q.ind, q.dist) for q in d2]
    assert len(profs) == maxL - minL + 1
    for j, p in enumerate(profs):
        m = minL + j
        assert p.shape == (len(x) - m + 1,)
        last = [e for e in log if e["m"] == m][-1]
        sel = p > -3e38
        assert int(sel.sum()) == last["n_cand"]
        assert p[d[j].ind] == np.float32(d[j].dist)
        nn, _ = O.nn_profile(x, m)
        assert np.all(np.abs(p[sel] - nn[sel]) <= 2 * m * 2e-4)


def test_cli_writes_range_discord_profile(tmp_path):
    import os
    import subprocess
    x = _series(8192, 5, "palmad")
    f = tmp_path / "ts.txt"
    np.savetxt(f, x, fmt="%.7g")
    exe = os.path.join(os.path.dirname(P.__file__), "paddi-main")
    prof = tmp_path / "profile.csv"
    r = subprocess.run([exe, str(f), str(len(x)), "40", "42", str(tmp_path / "d.csv"),
                        str(tmp_path / "t.csv"), "--profile", str(prof)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    rows = prof.read_text().strip().split("\n")
    assert [int(row.split(";")[0]) for row in rows] == [40, 41, 42]
    for row, m in zip(rows, (40, 41, 42)):
        assert len(row.split(";")) == 1 + len(x) - m + 1


def test_palmad_fp32_and_auto_agree(ctx, ctx32):
    x = _series(8192, 9, "palmad")
    a, la = ctx.palmad(x, 48, 56)
    b, lb = ctx32.palmad(x, 48, 56)
    assert a == b
    assert [(e["n_cand"], e["n_disc"]) for e in la] == [(e["n_cand"], e["n_disc"]) for e in lb]


def test_large_series_kernels_agree(ctx, ctx32):
    """17.8M points (refine ranges of millions of windows, window indices near
    2^24): the tensor-core refine and the FP32 refine must agree exactly, the
    top discords must sit in planted anomalies and their distances must be
    the exact FP64 nn of the reported windows."""
    n = (1 << 24) + (1 << 20)
    m = 64
    x, meta = datagen.pd3_series(n=n, seed=21, n_anom=4, anom_len=96)
    a, la = ctx.pd3(x, m, top_k=3)
    b, lb = ctx32.pd3(x, m, top_k=3)
    assert [(d.ind, d.dist) for d in a] == [(d.ind, d.dist) for d in b]
    assert [(e["n_cand"], e["n_disc"]) for e in la] == [(e["n_cand"], e["n_disc"]) for e in lb]
    spans = [(s - m, s + L) for s, L in zip(meta["starts"], meta["lengths"])]
    assert len(a) == 3
    for d in a:
        assert any(lo < d.ind < hi for lo, hi in spans), d
        want, _ = O.window_nn(x, m, d.ind)
        assert _close(d.dist, want)


# ------------------------------------------------------------------ edge cases
def test_flat_windows(ctx):
    rng = np.random.default_rng(7)
    x = np.cumsum(rng.standard_normal(6000)).astype(np.float32)
    x[1000:1100] = x[1000]          # flat run longer than 2m-1 for m=40
    x[3000:3050] = x[3000]          # a shorter flat run
    x[4500:4560] = np.float32(2.5)  # another flat run with a different level
    for m in (24, 40):
        want, watt = O.pd3(x, m, top_k=2)
        got, log = ctx.pd3(x, m, top_k=2)
        assert [d.ind for d in got] == [w[0] for w in want]
        for d, w in zip(got, want):
            assert _close(d.dist, w[1])
        assert [(e["n_cand"], e["n_disc"]) for e in log] == \
            [(e["n_cand"], e["n_disc"]) for e in watt]


def test_shortest_series(ctx):
    rng = np.random.default_rng(1)
    m = 50
    x = np.cumsum(rng.standard_normal(2 * m)).astype(np.float32)
    want, _ = O.pd3(x, m, top_k=1)
    got, _ = ctx.pd3(x, m, top_k=1)
    assert [d.ind for d in got] == [w[0] for w in want]


def test_threshold_exactly_at_a_distance(ctx32):
    x = _series(4096, 21)
    m = 48
    nn, _ = O.nn_profile(x, m)
    top = int(np.argmax(nn))
    # r2 equal to the float of the top distance: top is a candidate (nn >= r2)
    # but not a discord (nn > r2 fails)
    r2 = np.float32(nn[top])
    r = np.sqrt(r2, dtype=np.float32)
    while np.float32(r) * np.float32(r) != r2:  # find r with r*r == r2 in float
        r = np.nextafter(r, np.float32(np.inf) if r * r < r2 else np.float32(0))
        if abs(float(r * r) - float(r2)) > 1e-3 * float(r2):
            pytest.skip("no float r with r*r == nn")
    att, sel = O.select(nn, m, float(r2), top_k=1)
    got, log = ctx32.pd3(x, m, top_k=1, r=float(r))
    assert (log[0]["n_cand"], log[0]["n_disc"]) == (att["n_cand"], att["n_disc"])
    assert [d.ind for d in got] == [s[0] for s in sel]


def test_do_pd3_flags(ctx):
    import torch
    x = _series(6000, 33)
    m = 64
    nn, _ = O.nn_profile(x, m)
    r2 = float(np.float32(np.quantile(nn, 0.995)))
    N = len(x) - m + 1
    dT = torch.from_numpy(x).cuda()
    cand = torch.full((N,), -7, dtype=torch.int32, device="cuda")
    nnd = torch.zeros(N, dtype=torch.float32, device="cuda")
    nc = ctx.do_pd3(dT.data_ptr(), len(x), m, r2, cand.data_ptr(), nnd.data_ptr())
    torch.cuda.synchronize()
    want = (nn.astype(np.float32) >= np.float32(r2))
    got = cand.cpu().numpy().astype(bool)
    assert nc == int(want.sum())
    np.testing.assert_array_equal(got, want)
    d = nnd.cpu().numpy()
    np.testing.assert_allclose(d[want], nn[want], rtol=1e-3)
    assert np.all(d[~want] == -np.finfo(np.float32).max)


def test_invalid_arguments_return_status(ctx):
    x = _series(1000, 1)
    with pytest.raises(P.PaddiError) as e:
        ctx.pd3(x, 600)          # n < 2m
    assert e.value.status == P.PADDI_ERR_INVALID_ARG
    with pytest.raises(P.PaddiError) as e:
        ctx.palmad(x, 40, 30)    # maxL < minL
    assert e.value.status == P.PADDI_ERR_INVALID_ARG
    with pytest.raises(P.PaddiError):
        ctx.pd3(x, 32, top_k=99)


# ------------------------------------------------- every refine kernel, same answers
@pytest.mark.parametrize("dist", ["fp32", "fp16", "bf16"])
@pytest.mark.parametrize("n,m", [(8192, 64), (20000, 200), (12000, 361), (12000, 362),
                                 (16000, 500), (9000, 729)])
def test_refine_kernels_match_oracle(dist, n, m):
    dk = {"fp32": P.DIST_FP32, "fp16": P.DIST_SPLIT_FP16, "bf16": P.DIST_SPLIT_BF16}[dist]
    x = _series(n, 100 + m)
    nn, _ = O.nn_profile(x, m)
    with P.Context(distance_kernel=dk) as c:
        for q in (0.99, 0.9995):
            r2 = float(np.float32(np.quantile(nn, q)))
            r = float(np.sqrt(np.float32(r2)))
            r2f = np.float32(r) * np.float32(r)
            att, sel = O.select(nn, m, float(r2f), top_k=2)
            got, log = c.pd3(x, m, top_k=2, r=r)
            assert log[0]["refine_kernel"] == dk
            assert (log[0]["n_cand"], log[0]["n_disc"]) == (att["n_cand"], att["n_disc"])
            assert [d.ind for d in got] == [s[0] for s in sel]
            for d, s in zip(got, sel):
                assert _close(d.dist, s[1])


@pytest.mark.parametrize("dist", ["fp16", "bf16"])
@pytest.mark.parametrize("n,m", [(8192, 64), (20000, 200), (12000, 361)])
def test_refine_with_64_row_tiles_matches_oracle(dist, n, m):
    """The refine's tile rows forced to 64 (8 candidates per tile) where the
    length would pick 128: same counts and discords."""
    dk = {"fp16": P.DIST_SPLIT_FP16, "bf16": P.DIST_SPLIT_BF16}[dist]
    x = _series(n, 100 + m)
    nn, _ = O.nn_profile(x, m)
    with P.Context(distance_kernel=dk, tile_rows=64) as c:
        r2 = float(np.float32(np.quantile(nn, 0.995)))
        r = float(np.sqrt(np.float32(r2)))
        att, sel = O.select(nn, m, float(np.float32(r) * np.float32(r)), top_k=2)
        got, log = c.pd3(x, m, top_k=2, r=r)
        assert (log[0]["n_cand"], log[0]["n_disc"]) == (att["n_cand"], att["n_disc"])
        assert [d.ind for d in got] == [s[0] for s in sel]
        for d, s in zip(got, sel):
            assert _close(d.dist, s[1])


# -------------------------------------------- r policies change work, not results
@pytest.mark.parametrize("policy", ["bound"])
def test_r_policy_gives_the_same_discords(policy):
    rp = {"bound": P.R_BOUND}[policy]
    x = _series(8192, 5, "palmad")
    want, _ = O.palmad(x, 40, 60)
    with P.Context(r_policy=rp) as c:
        got, log = c.palmad(x, 40, 60)
    assert [d.ind for d in got] == [w[0] for w in want]
    for d, w in zip(got, want):
        assert _close(d.dist, w[1])
    # a guided attempt uses r^2 below a proven lower bound: it always succeeds
    guided = [e for e in log if e["r_source"] == 2]
    assert guided and all(e["found"] for e in guided)



def test_bound_is_the_exact_nn_of_the_previous_top_window():
    """The bound of every guided length is the exact FP64 nn, at that length,
    of the previous length's top-1 window.  On this series the top-1 window
    stays, moves by one or two places and jumps between anomalies, so the
    incremental dot products are reused, slid and rebuilt; a run on another
    series first must leave no state behind."""
    x = _series(8192, 5, "palmad")
    other = _series(8192, 6, "palmad")
    minL, maxL = 40, 70
    with P.Context(r_policy=P.R_BOUND) as c:
        c.palmad(other, minL, maxL)
        got, log = c.palmad(x, minL, maxL)
    want, _ = O.palmad(x, minL, maxL)
    assert [d.ind for d in got] == [w[0] for w in want]
    first = {}
    for e in log:
        first.setdefault(e["m"], e)
    checked = 0
    for m in range(minL + 1, maxL + 1):
        N = len(x) - m + 1
        w = min(got[m - 1 - minL].ind, N - 1)
        nn, _ = O.window_nn(x, m, w)
        lb = first[m]["lb"]
        if lb > 0:
            assert lb == float(np.float32(nn)), (m, w, lb, nn)
            checked += 1
    assert checked >= maxL - minL - 2


def test_guided_policies_report_merlins_distances_on_a_long_random_walk():
    """A held-out evaluation series (n = 2^20) whose top-1 windows have
    nearest neighbours at a series level far from their own: the bound
    window's nn, kept incrementally by the guided policies, must round to
    the same float as the recheck's direct FP64 value (lengths 530 and 567
    once differed by one unit in the last place)."""
    x = datagen.training_series(10, 1 << 20, 97, min_len=64, max_len=1024)[9]
    minL, maxL = 524, 572
    runs = {}
    for pol in (P.R_MERLIN, P.R_BOUND, P.R_LEARNED):
        with P.Context(r_policy=pol) as c:
            d, _ = c.palmad(x, minL, maxL)
        runs[pol] = [(q.ind, q.dist) for q in d]
    assert runs[P.R_BOUND] == runs[P.R_MERLIN]
    assert runs[P.R_LEARNED] == runs[P.R_MERLIN]
    exact = O.lengths_nn(x, minL, maxL, [w for w, _ in runs[P.R_MERLIN]])
    bad = [(minL + q, runs[P.R_MERLIN][q], e) for q, e in enumerate(exact)
           if float(np.float32(e)) != runs[P.R_MERLIN][q][1]]
    assert not bad, bad[:4]

# ------------------------------------------------------------- batched series
def test_batched_uneven_series_match_single_runs(ctx):
    series = [x for x, _ in datagen.batch_series(count=6, seed=3, min_log2=12, max_log2=13,
                                                 min_anom=32, max_anom=64)]
    minL, maxL = 32, 40
    got, att = ctx.palmad_batched(series, minL, maxL, streams=3)
    for x, g in zip(series, got):
        want, _ = O.palmad(x, minL, maxL)
        assert [d.ind for d in g] == [w[0] for w in want]
        for d, w in zip(g, want):
            assert _close(d.dist, w[1])
    assert all(a >= maxL - minL + 1 for a in att)


def test_batched_rejects_short_series(ctx):
    with pytest.raises(P.PaddiError) as e:
        ctx.palmad_batched([np.zeros(50, np.float32)], 32, 40)
    assert e.value.status == P.PADDI_ERR_INVALID_ARG


# ---------------------------------------------------------------------- CLI
def test_cli_writes_reference_csv_formats(tmp_path):
    import os
    import subprocess
    x = _series(6000, 8, "palmad")
    f = tmp_path / "series.txt"
    np.savetxt(f, x, fmt="%.6f")
    xr = np.loadtxt(f).astype(np.float32)  # the values the CLI reads
    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                       "paddi_b200", "paddi-main")
    d, t = tmp_path / "d.csv", tmp_path / "t.csv"
    r = subprocess.run([exe, str(f), str(len(x)), "40", "46", str(d), str(t)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lines = d.read_text().splitlines()
    assert lines[0] == "m;top-1 discord idx;top-1 discord nnDist"
    want, watt = O.palmad(xr, 40, 46)
    for line, w, m in zip(lines[1:], want, range(40, 47)):
        mm, ind, dist = line.split(";")
        assert (int(mm), int(ind)) == (m, w[0])
        assert abs(float(dist) - w[1]) <= 1e-4 * w[1]
    tl = t.read_text().splitlines()
    assert len(tl[0].split(";")) == 14 and len(tl) == 1 + len(watt)


# ------------------------------------------------------------------ autotuner
def test_autotune_picks_a_config_and_keeps_results():
    x = _series(20000, 12, "palmad")
    with P.Context() as c:
        cfg = c.autotune(x, 48, 60)
        assert cfg["segment_len"] in (256, 384, 512) and cfg["phase1_chunks"] in (8, 12, 16)
        assert cfg["tile_rows"] in (0, 64)
        assert len(cfg["probe_ms"]) == 18
        assert all(v > 0 for v in cfg["probe_ms"].values())
        got, _ = c.palmad(x, 48, 60)
    want, _ = O.palmad(x, 48, 60)
    assert [d.ind for d in got] == [w[0] for w in want]


@pytest.mark.slow
def test_batched_workload_sample_properties():
    # a slice of the batched workload (uneven series, L=32..64): the batched
    # call equals one call per series, and each reported top-1 carries its
    # exact FP64 nearest-neighbour distance
    series = [x for x, _ in datagen.batch_series(count=12, seed=2, min_log2=14, max_log2=16)]
    minL, maxL = 32, 64
    with P.Context(r_policy=P.R_LEARNED) as c:
        got, _ = c.palmad_batched(series, minL, maxL, streams=4)
        one = [c.palmad(x, minL, maxL)[0] for x in series[:3]]
    assert got[:3] == one
    rng = np.random.default_rng(0)
    for x, g in zip(series, got):
        for i in rng.choice(maxL - minL + 1, 2, replace=False):
            d, _ = O.window_nn(x, minL + i, g[i].ind)
            assert abs(g[i].dist - d) <= 1e-5 * d


@pytest.mark.parametrize("far_partner", [False, True])
def test_flat_window_span(ctx, far_partner):
    """Flat windows with and without an admissible flat partner.

    A flat run of m+5 values gives 6 flat windows, all closer than m-1 to
    each other: each one's nearest neighbour is a non-flat window at d = 2m,
    so they lead the discord list.  A second flat run far away gives every
    flat window a partner at d = 0; those are dropped at candidate compaction.
    """
    rng = np.random.default_rng(11)
    m = 40
    x = np.cumsum(rng.standard_normal(20000)).astype(np.float32)
    x[5000:5000 + m + 5] = x[5000]
    if far_partner:
        x[15000:15060] = np.float32(-3.0)
    want, watt = O.pd3(x, m, top_k=3)
    got, log = ctx.pd3(x, m, top_k=3)
    assert [d.ind for d in got] == [w[0] for w in want]
    for d, w in zip(got, want):
        assert _close(d.dist, w[1])
    assert [(e["n_cand"], e["n_disc"]) for e in log] == \
        [(e["n_cand"], e["n_disc"]) for e in watt]
    # fixed thresholds: a tiny r (inside the guard band of rho = 1), r^2 just
    # below 2m (the flat windows without a partner stay) and just above it
    # (flat vs non-flat pairs, d = 2m, prune)
    nn, _ = O.nn_profile(x, m)
    for r in (0.05, 1.0, float(np.sqrt(2.0 * m)) - 0.1, float(np.sqrt(2.0 * m)) + 0.5):
        r2 = float(np.float32(r) * np.float32(r))
        att, sel = O.select(nn, m, r2, top_k=3)
        g, lg = ctx.pd3(x, m, top_k=3, r=r)
        assert (lg[0]["n_cand"], lg[0]["n_disc"]) == (att["n_cand"], att["n_disc"]), r
        assert [d.ind for d in g] == [s[0] for s in sel], r
