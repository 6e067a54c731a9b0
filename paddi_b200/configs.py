"""Timing runs of the reference's other configurations on seeded synthetic data.

    python -m paddi_b200.configs fixed      # C1: PD3, n = 131072, m = 128, segment 4096, top-4
    python -m paddi_b200.configs batched    # C3: 256 series of 2^14..2^18 points, lengths 32..256
    python -m paddi_b200.configs all

C1 follows the reference's fixed-length run (src/main.cu:136-156: r halved
from 2 sqrt(m) until the discords are found, top-k as hinted at :137) with
its segment length (SEGMENT_N, src/parameters.hpp:8-10) set to 4096, and
also with this library's default segment of 256 rows.  C3 runs
``paddi_palmad_batched`` (worker contexts on 4 streams) under the MERLIN and
the learned r policies and checks that both give the same discords.  Each
prints one JSON line; times are device time (CUDA events on the context's
stream) for C1 and wall time of the batched call for C3.
"""
from __future__ import annotations

import argparse
import json
import time

from . import R_LEARNED, R_MERLIN, Context
from . import datagen


def fixed_length(reps: int = 5):
    import torch
    x, _ = datagen.pd3_series(n=131072, seed=0)
    out = {"config": "PD3 n=131072 m=128 top-4, r halved from 2 sqrt(m)"}
    with Context(device=0) as ctx:
        ctx.pd3(x, 128, top_k=4, segment_len=4096)  # warm
        st = torch.cuda.ExternalStream(ctx.stream)
        for seg in (4096, 256):
            ts = []
            for _ in range(reps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(st)
                d, log = ctx.pd3(x, 128, top_k=4, segment_len=seg)
                e1.record(st)
                e1.synchronize()
                ts.append(e0.elapsed_time(e1))
            out[f"segment_{seg}"] = {"ms_median": sorted(ts)[len(ts) // 2],
                                     "attempts": len(log),
                                     "discords": [(q.ind, q.dist) for q in d]}
    return out


def batched(streams: int = 4):
    series = [s for s, _ in datagen.batch_series(256, seed=2)]
    out = {"config": f"256 series of 2^14..2^18 points, lengths 32..256, {streams} streams"}
    ref = None
    for name, pol in (("merlin", R_MERLIN), ("learned", R_LEARNED)):
        with Context(device=0, r_policy=pol) as ctx:
            ctx.palmad_batched(series[:4], 32, 40, streams=streams)  # warm
            t = time.perf_counter()
            disc, att = ctx.palmad_batched(series, 32, 256, streams=streams)
            sec = time.perf_counter() - t
        got = [[(q.ind, q.dist) for q in d] for d in disc]
        ref = got if ref is None else ref
        out[name] = {"s": sec, "attempts": int(sum(att)), "same_discords": got == ref}
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("which", choices=["fixed", "batched", "all"])
    a = ap.parse_args(argv)
    if a.which in ("fixed", "all"):
        print(json.dumps(fixed_length()), flush=True)
    if a.which in ("batched", "all"):
        print(json.dumps(batched()), flush=True)


if __name__ == "__main__":
    main()
