#!/usr/bin/env python3
"""Generates the golden fixtures of tests/golden/ from the reference itself.

The reference ships no tests, fixtures or golden vectors, so the fixtures
are outputs of its own CPU kernels (src/cpu_kernels/cpu_kernels.cpp,
compiled unmodified into oracle/_ref/libpaddi_ref.so by oracle/Makefile)
on seeded synthetic inputs:

  ref_stats.npz       compute_statistics_cpu  (mean, std)  for three lengths
  ref_attempts.npz    find_discords_cpu       (candidate flags, nnDist) for
                      several (m, r) on two series, plus the attempt record
                      (candidates, discords, top-1) of the restated driver
  ref_palmad.json     the MERLIN-scheduled PALMAD run of the reference CPU
                      path (src/main.cu:136-233 restated around the kernels)
  oracle_palmad.json  the FP64 oracle's PALMAD on the same series with the
                      GPU exclusion rule (regression fixture for the oracle)

Run from the repository root:  python tests/golden/make_golden.py
It needs the reference sources (to build oracle/_ref); the tests only read
the files written here.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from paddi_b200 import datagen  # noqa: E402


def series_a():
    x, _ = datagen.pd3_series(n=3000, seed=11, n_anom=3, anom_len=60)
    return x


def series_b():
    """Random walk + sinusoid with a noise and a time-reversal anomaly (no
    flatline: the reference's FP32 statistics of a constant window are
    rounding noise, a case the oracle settles by policy instead)."""
    rng = np.random.default_rng(12)
    x = datagen.random_walk_sine(2500, rng)
    datagen.plant_anomalies(x, [700, 1600], [48, 60], ["noise", "reverse"], rng)
    return x.astype(np.float32)


def main():
    O.build()
    x = series_a()
    st = {}
    for m in (8, 32, 100):
        mu, sd = O.ref_statistics(x, m)
        st[f"mean_{m}"] = mu
        st[f"std_{m}"] = sd
    np.savez_compressed(os.path.join(HERE, "ref_stats.npz"), x=x, **st)

    att = {}
    meta = []
    for name, s in (("a", series_a()), ("b", series_b())):
        att[f"x_{name}"] = s
        for m in (16, 50):
            for r in (2.0 * np.sqrt(m) / 2.0, 2.0 * np.sqrt(m) / 3.0, 2.0 * np.sqrt(m) / 4.0):
                r = float(np.float32(r))
                a, cand, nnd = O.ref_attempt(s, m, r)
                key = f"{name}_{m}_{len(meta)}"
                att[f"cand_{key}"] = cand
                att[f"nnd_{key}"] = nnd
                meta.append({"key": key, "series": name, "m": m, "r": r, **a})
    np.savez_compressed(os.path.join(HERE, "ref_attempts.npz"), **att)
    with open(os.path.join(HERE, "ref_attempts.json"), "w") as f:
        json.dump(meta, f, indent=1)

    xp = series_b()
    disc, log = O.ref_palmad(xp, 24, 33)
    with open(os.path.join(HERE, "ref_palmad.json"), "w") as f:
        json.dump({"series": "series_b", "minL": 24, "maxL": 33,
                   "discords": disc, "attempts": log}, f, indent=1)

    disc, log = O.palmad(xp, 24, 33)
    with open(os.path.join(HERE, "oracle_palmad.json"), "w") as f:
        json.dump({"series": "series_b", "minL": 24, "maxL": 33,
                   "discords": disc, "attempts": log}, f, indent=1)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()
