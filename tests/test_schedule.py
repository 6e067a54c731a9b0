"""The library's MERLIN r-schedule (pure host code, no GPU needed) against the
reference's own CPU run.

``tests/golden/ref_palmad.json`` records every attempt of a PALMAD run of the
reference's CPU kernels (src/cpu_kernels/cpu_kernels.cpp) under its MERLIN
schedule (src/main.cu:136-233).  Replaying that run's top-1 distances through
``paddi_merlin_first_r`` / ``paddi_merlin_lower`` must give the reference's
threshold at every attempt, bit for bit.
"""
import json
import os

import numpy as np

from paddi_b200 import sharded

HERE = os.path.dirname(os.path.abspath(__file__))


def test_exported_merlin_schedule_replays_the_reference_run():
    g = json.load(open(os.path.join(HERE, "golden", "ref_palmad.json")))
    minL, maxL = g["minL"], g["maxL"]
    by_m = {}
    for a in g["attempts"]:
        by_m.setdefault(a["m"], []).append(a)
    out = []
    checked = 0
    for j in range(maxL - minL + 1):
        m = minL + j
        r, S = sharded.merlin_first_r(out, j, minL)
        for a in by_m[m]:
            assert np.float32(r) == np.float32(a["r"]), (m, r, a["r"])
            checked += 1
            if a["found"]:
                break
            r = sharded.merlin_lower(r, j, S)
        ind, dist = g["discords"][j]
        out.append((ind, dist))
    assert checked == len(g["attempts"])
