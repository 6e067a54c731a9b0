"""Learned r for PALMAD: data, training recipe and the bundled model.

The predictor (kernels in csrc/k_mlp.cu, ABI paddi_model_*) estimates
y = log(d_m / d_{m-1}), the growth of the top-1 squared discord distance from
length m-1 to m, from 12 features of the previous lengths
(paddi_r_features).  It is trained with the pinball loss at a low quantile,
so r^2 = d_{m-1} exp(y_hat) tends to sit just below the true distance.

Training data are the method's own logs: plain MERLIN PALMAD runs
(PADDI_FLAG_LOG_BOUND so the bound feature is logged too) over seeded series
from ``datagen.training_series``.  A wrong prediction never changes the
discords, only the number of attempts.

Recipe of the bundled model (GPU; collecting the logs of 512 MERLIN runs on
series of 2^18 points at lengths 64..1024 takes ~14 minutes on a B200, the
training a few seconds):
    python -m paddi_b200.learned_r train --series 512 --n 262144 --minL 64 --maxL 1024 --seed 31 --tau 0.1
writes paddi_b200/models/r_mlp.npz; ``load_default`` reads it (``--save-samples``
keeps the collected pairs, ``--samples`` trains from them again).  Evaluation
on held-out series (another seed), all three r policies:
    python -m paddi_b200.learned_r evaluate --series 64 --n 1048576 --minL 64 --maxL 1024 --seed 97
"""
from __future__ import annotations

import argparse
import os
import time

import numpy as np

from . import (DIST_AUTO, FLAG_LOG_BOUND, MODEL_NPARAM, PADDI_ERR_ITER_CAP, R_LEARNED,
               R_MERLIN, Context, PaddiError, init_params, r_features)
from . import datagen

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_MODEL = os.path.join(HERE, "models", "r_mlp.npz")


def load_default():
    """Parameters of the bundled model (raises if it was not trained yet)."""
    d = np.load(DEFAULT_MODEL)
    p = d["params"].astype(np.float32)
    assert p.size == MODEL_NPARAM
    return p


def log_features(discords, log, minL: int):
    """(X, Y) training pairs from one PALMAD run: one row per length >= minL+1.

    discords: [(ind, dist)] per length; log: attempt rows (dicts) of the run.
    """
    by_m = {}
    for e in log:
        by_m.setdefault(e["m"], []).append(e)
    X, Y = [], []
    prev_attempts = 0
    for j, (ind, dist) in enumerate(discords):
        m = minL + j
        rows = by_m.get(m, [])
        if j >= 1 and rows and dist > 0 and discords[j - 1][1] > 0:
            first = rows[0]
            f = r_features(discords, j, minL, first["lb"], first["flat_frac"], prev_attempts)
            X.append(f)
            Y.append(np.log(dist / discords[j - 1][1]))
        prev_attempts = len(rows)
    return np.array(X, np.float32).reshape(-1, 12), np.array(Y, np.float32)


def collect(series_list, minL, maxL, device=0):
    """Plain MERLIN runs with the bound logged; returns X, Y and run stats.

    A series on which plain MERLIN does not converge (its decrement S of
    src/main.cu:230 vanishes; the reference would loop forever) is skipped
    and counted in the stats as "skipped".
    """
    Xs, Ys, runs = [], [], []
    with Context(device=device, distance_kernel=DIST_AUTO, r_policy=R_MERLIN,
                 flags=FLAG_LOG_BOUND) as ctx:
        for x in series_list:
            t = time.perf_counter()
            try:
                d, log = ctx.palmad(x, minL, maxL)
            except PaddiError as e:
                if e.status != PADDI_ERR_ITER_CAP:
                    raise
                runs.append({"s": time.perf_counter() - t, "skipped": True})
                continue
            runs.append({"s": time.perf_counter() - t, "attempts": len(log)})
            X, Y = log_features([(q.ind, q.dist) for q in d], log, minL)
            Xs.append(X)
            Ys.append(Y)
    return np.concatenate(Xs), np.concatenate(Ys), runs


def train(X, Y, tau=0.2, epochs=300, batch=2048, lr=2e-3, seed=0, device=0):
    with Context(device=device) as ctx:
        return ctx.model_train(X, Y, tau=tau, epochs=epochs, batch=batch, lr=lr, seed=seed,
                               init=init_params(seed))


def compare(series_list, minL, maxL, params, margin=1.0, device=0):
    """Attempts and time per series: plain MERLIN vs the learned policy."""
    rows = []
    for x in series_list:
        rec = {}
        for name, pol in (("merlin", R_MERLIN), ("learned", R_LEARNED)):
            kw = {"model": params, "model_margin": margin} if pol == R_LEARNED else {}
            with Context(device=device, r_policy=pol, **kw) as ctx:
                ctx.palmad(x, minL, minL + 4)  # warm
                t = time.perf_counter()
                d, log = ctx.palmad(x, minL, maxL)
                rec[name] = {"s": time.perf_counter() - t, "attempts": len(log),
                             "discords": [(q.ind, q.dist) for q in d],
                             "ms": sum(e["ms_total"] for e in log)}
        rows.append(rec)
    return rows


def evaluate(series_list, minL, maxL, device=0, model=None, policies=("merlin", "bound", "learned"),
             margin=1.0):
    """Attempts and seconds per series for the MERLIN, BOUND and LEARNED
    policies (same kernels); checks that the discords are identical.  A
    policy that reaches the attempt cap on a series (plain MERLIN can: its
    decrement S of src/main.cu:230 may vanish) is recorded as None."""
    from . import R_BOUND
    codes = {"merlin": R_MERLIN, "bound": R_BOUND, "learned": R_LEARNED}
    rows = []
    for x in series_list:
        rec, ref = {}, None
        for name in policies:
            pol = codes[name]
            kw = {}
            if pol == R_LEARNED:
                kw["model_margin"] = margin
                if model is not None:
                    kw["model"] = model
            with Context(device=device, r_policy=pol, **kw) as ctx:
                ctx.palmad(x, minL, minL + 2)  # warm
                t = time.perf_counter()
                try:
                    d, log = ctx.palmad(x, minL, maxL)
                except PaddiError as e:
                    if e.status != PADDI_ERR_ITER_CAP:
                        raise
                    rec[name] = None
                    continue
                disc = [(q.ind, q.dist) for q in d]
                ref = disc if ref is None else ref
                rec[name] = {"s": time.perf_counter() - t, "attempts": len(log),
                             "same": disc == ref}
        rows.append(rec)
    return rows


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("cmd", choices=["train", "evaluate"])
    ap.add_argument("--series", type=int, default=64)
    ap.add_argument("--n", type=int, default=1 << 17)
    ap.add_argument("--minL", type=int, default=64)
    ap.add_argument("--maxL", type=int, default=512)
    ap.add_argument("--seed", type=int, default=31)
    ap.add_argument("--tau", type=float, default=0.1)
    ap.add_argument("--epochs", type=int, default=300)
    ap.add_argument("--out", default=DEFAULT_MODEL)
    ap.add_argument("--model", default=None, help="evaluate: model file (default: the bundled one)")
    ap.add_argument("--json", default=None, help="evaluate: write the per-series rows here")
    ap.add_argument("--policies", default="merlin,bound,learned",
                    help="evaluate: comma-separated subset of merlin,bound,learned")
    ap.add_argument("--margin", type=float, default=1.0,
                    help="evaluate: scale of the model's predicted r^2")
    ap.add_argument("--first", type=int, default=0,
                    help="evaluate: only the first this many series (0: all)")
    ap.add_argument("--save-samples", default=None,
                    help="train: also write the collected (X, Y) pairs to this .npz")
    ap.add_argument("--samples", default=None,
                    help="train: read (X, Y) pairs from this .npz instead of collecting them")
    a = ap.parse_args(argv)
    if a.cmd == "train" and a.samples:
        series = []
    else:
        series = datagen.training_series(a.series, a.n, a.seed, min_len=a.minL, max_len=a.maxL)
    if a.cmd == "evaluate":
        model = None
        if a.model:
            model = np.load(a.model)["params"].astype(np.float32)
        if a.first:
            series = series[:a.first]
        pols = tuple(p for p in a.policies.split(",") if p)
        rows = evaluate(series, a.minL, a.maxL, model=model, policies=pols, margin=a.margin)
        if a.json:
            import json
            with open(a.json, "w") as fh:
                json.dump({"series": len(rows), "n": a.n, "minL": a.minL, "maxL": a.maxL,
                           "seed": a.seed, "model": a.model or DEFAULT_MODEL,
                           "margin": a.margin, "rows": rows}, fh)
        L = a.maxL - a.minL + 1
        ok = [r for r in rows if all(r[p] is not None for p in r)]
        capped_m = sum(1 for r in rows if "merlin" in r and r["merlin"] is None)
        print(f"series {len(rows)}; plain MERLIN reached the attempt cap on "
              f"{capped_m}; totals over the other {len(ok)}")
        for name in pols:
            att = sum(r[name]["attempts"] for r in ok)
            sec = sum(r[name]["s"] for r in ok)
            same = all(r[name]["same"] for r in ok)
            capped = sum(1 for r in rows if r[name] is None)
            print(f"{name:8s} attempts/length {att / (L * max(1, len(ok))):.3f}  seconds {sec:.2f}  "
                  f"same discords {same}  capped {capped}")
        return
    t = time.perf_counter()
    if a.samples:
        d = np.load(a.samples)
        X, Y = d["X"].astype(np.float32), d["Y"].astype(np.float32)
        runs = [{"skipped": bool(v)} for v in d["skipped"]]
    else:
        X, Y, runs = collect(series, a.minL, a.maxL)
        if a.save_samples:
            np.savez_compressed(a.save_samples, X=X, Y=Y,
                                skipped=np.array([bool(r.get("skipped")) for r in runs]))
    t_collect = time.perf_counter() - t
    t = time.perf_counter()
    params, loss = train(X, Y, tau=a.tau, epochs=a.epochs)
    t_train = time.perf_counter() - t
    os.makedirs(os.path.dirname(a.out), exist_ok=True)
    np.savez_compressed(a.out, params=params, loss=loss, tau=a.tau,
                        recipe=np.array(f"series={a.series} n={a.n} L={a.minL}..{a.maxL} "
                                        f"seed={a.seed} tau={a.tau} epochs={a.epochs}"))
    skipped = sum(1 for r in runs if r.get("skipped"))
    print(f"samples={len(Y)} series={len(runs)} skipped={skipped} "
          f"collect={t_collect:.1f}s train={t_train:.1f}s "
          f"loss {loss[0]:.4f} -> {loss[-1]:.4f}; wrote {a.out}")


if __name__ == "__main__":
    main()
