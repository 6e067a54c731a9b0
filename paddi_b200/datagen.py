"""Seeded synthetic series for the five discord-discovery workloads.

The reference's runners read datasets (ECG, RandomWalk, MGAB, GAP/ASTRO,
power_demand, Bearing: src/runners/**.sbatch) that are not shipped with it.
These generators stand in for them with the same shapes and value
distributions; every series is float32 and fully determined by its seed
(numpy PCG64).

Workloads
---------
* ``pd3_series``     one random walk + sinusoid, 4 planted noise windows
                     (fixed-length PD3, n = 131072, m = 128).
* ``palmad_series``  the same generator with 16 planted anomalies of three
                     kinds: noise, flatline, time reversal
                     (PALMAD, n = 2^21, L = 64..512).
* ``batch_series``   256 uneven series, lengths U[2^14, 2^18], each a random
                     walk + sinusoid mix with 1-3 anomalies of length 32-256.
* ``ecg_series``     ECG-like beats (Gaussian bumps, period 250 +/- 20) with
                     noise, baseline wander and morphologically altered beats.
* ``hostile_series`` series built to stress FP32 / 16-bit rounding: near-flat
                     stretches, a large offset with unit local variance,
                     integer-quantised values with many ties.

Anomaly positions never overlap; every generator returns the planted
positions so tests can check that discords land on them.
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "random_walk_sine",
    "plant_anomalies",
    "pd3_series",
    "palmad_series",
    "batch_series",
    "ecg_series",
    "training_series",
    "hostile_series",
]


def random_walk_sine(n: int, rng: np.random.Generator, period: float = 200.0,
                     amp: float = 0.5) -> np.ndarray:
    """cumsum(N(0,1)) + amp*sin(2*pi*t/period), computed in float64."""
    t = np.arange(n, dtype=np.float64)
    return np.cumsum(rng.standard_normal(n)) + amp * np.sin(2.0 * np.pi * t / period)


def _non_overlapping_starts(n: int, lengths, rng: np.random.Generator,
                            margin: int = 0) -> list[int]:
    """Pick one start per length so that the planted windows do not overlap.

    Rejection sampling on [margin, n - L - margin); deterministic for a seed.
    """
    starts: list[int] = []
    taken: list[tuple[int, int]] = []
    for L in lengths:
        for _ in range(10000):
            s = int(rng.integers(margin, n - L - margin))
            if all(s + L <= a or b <= s for a, b in taken):
                break
        else:  # pragma: no cover - only for absurdly dense requests
            raise ValueError("cannot place non-overlapping anomalies")
        starts.append(s)
        taken.append((s, s + L))
    return starts


def plant_anomalies(x: np.ndarray, starts, lengths, kinds,
                    rng: np.random.Generator, noise_std: float = 3.0) -> None:
    """Overwrite ``x`` in place.

    kinds: 'noise'   -> the window is replaced by N(0, noise_std) samples
                        (std, not variance),
           'flat'    -> the window is replaced by its first value,
           'reverse' -> the window is time-reversed.
    """
    for s, L, k in zip(starts, lengths, kinds):
        if k == "noise":
            x[s:s + L] = rng.normal(0.0, noise_std, L)
        elif k == "flat":
            x[s:s + L] = x[s]
        elif k == "reverse":
            x[s:s + L] = x[s:s + L][::-1].copy()
        else:
            raise ValueError(k)


def pd3_series(n: int = 131072, seed: int = 0, n_anom: int = 4,
               anom_len: int = 150):
    """Fixed-length workload: random walk + 0.5 sin(2 pi t/200), seed 0,
    ``n_anom`` windows of ``anom_len`` points replaced by N(0,3) noise."""
    rng = np.random.default_rng(seed)
    x = random_walk_sine(n, rng)
    lengths = [anom_len] * n_anom
    starts = _non_overlapping_starts(n, lengths, rng, margin=anom_len)
    plant_anomalies(x, starts, lengths, ["noise"] * n_anom, rng)
    return x.astype(np.float32), {"starts": starts, "lengths": lengths,
                                  "kinds": ["noise"] * n_anom}


def palmad_series(n: int = 1 << 21, seed: int = 1, n_anom: int = 16,
                  min_len: int = 64, max_len: int = 512,
                  kinds_cycle=("noise", "flat", "reverse")):
    """Arbitrary-length workload: same generator, ``n_anom`` anomalies with
    lengths U[min_len, max_len] cycling through ``kinds_cycle``."""
    rng = np.random.default_rng(seed)
    x = random_walk_sine(n, rng)
    lengths = [int(v) for v in rng.integers(min_len, max_len + 1, n_anom)]
    kinds = [kinds_cycle[i % len(kinds_cycle)] for i in range(n_anom)]
    starts = _non_overlapping_starts(n, lengths, rng, margin=max_len)
    plant_anomalies(x, starts, lengths, kinds, rng)
    return x.astype(np.float32), {"starts": starts, "lengths": lengths,
                                  "kinds": kinds}


def batch_series(count: int = 256, seed: int = 2, min_log2: int = 14,
                 max_log2: int = 18, min_anom: int = 32, max_anom: int = 256):
    """Uneven batch: ``count`` series, one seed each (seed*100003 + i)."""
    out = []
    for i in range(count):
        rng = np.random.default_rng(seed * 100003 + i)
        n = int(rng.integers(1 << min_log2, (1 << max_log2) + 1))
        period = float(rng.uniform(50.0, 400.0))
        x = random_walk_sine(n, rng, period=period, amp=float(rng.uniform(0.3, 2.0)))
        k = int(rng.integers(1, 4))
        lengths = [int(v) for v in rng.integers(min_anom, max_anom + 1, k)]
        kinds = [("noise", "flat", "reverse")[int(v)] for v in rng.integers(0, 3, k)]
        starts = _non_overlapping_starts(n, lengths, rng, margin=max_anom)
        plant_anomalies(x, starts, lengths, kinds, rng)
        out.append((x.astype(np.float32), {"starts": starts, "lengths": lengths,
                                           "kinds": kinds}))
    return out


def training_series(count: int, n: int, seed: int, min_anom_count: int = 4,
                    max_anom_count: int = 8, min_len: int = 64, max_len: int = 1024):
    """Series for learning the r predictor: random walk + sinusoid with
    ``min_anom_count``..``max_anom_count`` planted anomalies each."""
    out = []
    for i in range(count):
        rng = np.random.default_rng(seed * 7919 + i)
        x = random_walk_sine(n, rng, period=float(rng.uniform(50.0, 400.0)))
        k = int(rng.integers(min_anom_count, max_anom_count + 1))
        lengths = [int(v) for v in rng.integers(min_len, max_len + 1, k)]
        kinds = [("noise", "flat", "reverse")[int(v)] for v in rng.integers(0, 3, k)]
        starts = _non_overlapping_starts(n, lengths, rng, margin=max_len)
        plant_anomalies(x, starts, lengths, kinds, rng)
        out.append(x.astype(np.float32))
    return out


def ecg_series(n: int = 1 << 27, seed: int = 5, n_altered: int = 64,
               period: float = 250.0, jitter: float = 20.0):
    """ECG-like series: a Gaussian-bump beat template repeated with period
    ``period`` +/- U(jitter), N(0, 0.05) additive noise, a slow baseline
    wander of amplitude 0.3, and ``n_altered`` beats whose amplitude is
    scaled by U[0.4, 2] and width by U[0.5, 2]."""
    rng = np.random.default_rng(seed)
    # beat onsets
    n_beats = int(n / (period - jitter)) + 2
    gaps = period + rng.uniform(-jitter, jitter, n_beats)
    onsets = np.cumsum(gaps) - gaps[0]
    onsets = onsets[onsets < n]
    altered = set(int(v) for v in rng.choice(len(onsets), size=min(n_altered, len(onsets)),
                                             replace=False))
    amp = np.ones(len(onsets))
    width = np.ones(len(onsets))
    for b in altered:
        amp[b] = rng.uniform(0.4, 2.0)
        width[b] = rng.uniform(0.5, 2.0)
    # template: P wave, QRS complex, T wave as Gaussian bumps (offset, height, sigma)
    bumps = ((40.0, 0.15, 8.0), (90.0, -0.12, 3.0), (100.0, 1.0, 4.0),
             (110.0, -0.25, 3.5), (170.0, 0.3, 14.0))
    x = np.zeros(n, dtype=np.float64)
    span = 256

    def beat(tt, w):
        seg = np.zeros_like(tt)
        for off, h, sg in bumps:
            seg += h * np.exp(-0.5 * ((tt - off * w) / (sg * w)) ** 2)
        return seg

    # unaltered beats: vectorised in chunks; even and odd beats apart so that
    # no two beats of one scatter overlap (beats are >= 230 apart, 257 long)
    plain = np.array([b for b in range(len(onsets)) if b not in altered], dtype=np.int64)
    k = np.arange(span + 1, dtype=np.int64)
    for parity in (0, 1):
        idx = plain[plain % 2 == parity]
        for c0 in range(0, len(idx), 1 << 15):
            bb = idx[c0:c0 + (1 << 15)]
            a0 = onsets[bb].astype(np.int64)
            pos = a0[:, None] + k[None, :]
            tt = pos - onsets[bb][:, None]
            seg = amp[bb][:, None] * beat(tt, 1.0)
            ok = pos < n
            x[pos[ok]] += seg[ok]
    for b in sorted(altered):
        t0 = onsets[b]
        a0 = int(t0)
        a1 = min(n, a0 + int(span * width[b]) + 1)
        if a1 <= a0:
            continue
        tt = np.arange(a0, a1, dtype=np.float64) - t0
        x[a0:a1] += amp[b] * beat(tt, width[b])
    t = np.arange(n, dtype=np.float64)
    x += 0.3 * np.sin(2.0 * np.pi * t / 7919.0) + rng.normal(0.0, 0.05, n)
    return x.astype(np.float32), {"altered_onsets": sorted(int(onsets[b]) for b in altered)}


def hostile_series(kind: str, n: int = 1 << 14, seed: int = 0):
    """Series whose windows have a large |mean - tile level| / std ratio,
    the case where the distance kernels' rounding is amplified.

    kind: 'near_flat' -> random walk + sinusoid with 6 stretches of 300 points
                         whose values vary by about 1e-5 of the walk's range
                         around a level (N(0, 1e-5 * range) on the level);
          'offset'    -> 1e4 + sin(2 pi t/200) + N(0, 0.3): unit local
                         variance on a large offset, 4 noise anomalies;
          'quantised' -> round(2 * random walk) / 2 with 4 planted anomalies:
                         many ties, flat runs and near-flat windows;
          'ecg_flat'  -> the ECG-like generator with its beats removed from
                         4 stretches of 1500 points (a flat, slightly noisy
                         baseline).
    Returns (float32 series, info)."""
    rng = np.random.default_rng(seed)
    if kind == "near_flat":
        x = random_walk_sine(n, rng)
        span = float(x.max() - x.min())
        lengths = [300] * 6
        starts = _non_overlapping_starts(n, lengths, rng, margin=300)
        for s0 in starts:
            x[s0:s0 + 300] = x[s0] + rng.normal(0.0, 1e-5 * span, 300)
        return x.astype(np.float32), {"starts": starts, "lengths": lengths}
    if kind == "offset":
        t = np.arange(n, dtype=np.float64)
        x = 1e4 + np.sin(2.0 * np.pi * t / 200.0) + rng.normal(0.0, 0.3, n)
        lengths = [120] * 4
        starts = _non_overlapping_starts(n, lengths, rng, margin=120)
        for s0 in starts:
            x[s0:s0 + 120] = 1e4 + rng.normal(0.0, 1.5, 120)
        return x.astype(np.float32), {"starts": starts, "lengths": lengths}
    if kind == "quantised":
        x = random_walk_sine(n, rng)
        lengths = [100] * 4
        starts = _non_overlapping_starts(n, lengths, rng, margin=100)
        plant_anomalies(x, starts, lengths, ["noise", "flat", "reverse", "noise"], rng)
        return (np.round(2.0 * x) / 2.0).astype(np.float32), {"starts": starts,
                                                               "lengths": lengths}
    if kind == "ecg_flat":
        x, info = ecg_series(n=n, seed=seed, n_altered=4)
        x = x.astype(np.float64)
        base = np.median(x)
        lengths = [1500] * 4
        starts = _non_overlapping_starts(n, lengths, rng, margin=500)
        for s0 in starts:
            x[s0:s0 + 1500] = base + rng.normal(0.0, 1e-3, 1500)
        return x.astype(np.float32), {"starts": starts, "lengths": lengths}
    raise ValueError(kind)
