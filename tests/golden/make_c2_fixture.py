"""Fixture of the headline PALMAD configuration (n = 2^21, lengths 64..512).

Writes tests/golden/c2_top1.json: for selected lengths m, the top-1 discord of
the full FP64 nearest-neighbour profile of ``datagen.palmad_series(n=2**21,
seed=1)`` (oracle.nn_profile_fast: every window against every admissible
window, O(N^2) per length, several minutes per length on 8 cores).  The
PALMAD top-1 of a length is the first maximum of float(nn) (the discord rule
nn > r^2 with the final r below it, src/sets_processing.hpp:11-46), so the
GPU test compares the library's reported window and distance at these
lengths with these values.  A SHA-256 of the series bytes guards against a
change of the generator.

    python tests/golden/make_c2_fixture.py 64 65 288 512   # adds / replaces lengths
"""
import hashlib
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from oracle import oracle as O  # noqa: E402
from paddi_b200 import datagen  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "c2_top1.json")
N_SERIES, SEED = 1 << 21, 1


def main(lengths):
    x, _ = datagen.palmad_series(n=N_SERIES, seed=SEED)
    digest = hashlib.sha256(np.ascontiguousarray(x, np.float32).tobytes()).hexdigest()
    doc = {"series": f"datagen.palmad_series(n={N_SERIES}, seed={SEED})", "sha256": digest,
           "lengths": {}}
    if os.path.exists(OUT):
        old = json.load(open(OUT))
        if old.get("sha256") == digest:
            doc["lengths"] = old["lengths"]
    for m in lengths:
        t = time.time()
        nn = O.nn_profile_fast(x, m)
        i, d = O.top1(nn)
        f = nn.astype(np.float32)
        order = np.argsort(-f, kind="stable")
        # the best window that does not overlap the top-1 (|i - j| >= m - 1)
        far = next(int(j) for j in order if abs(int(j) - i) >= m - 1)
        doc["lengths"][str(m)] = {"ind": i, "dist": d, "nn64": float(nn[i]),
                                  "next_nonoverlapping": [far, float(f[far])],
                                  "seconds": round(time.time() - t, 1)}
        print(m, doc["lengths"][str(m)], flush=True)
        with open(OUT, "w") as fh:
            json.dump(doc, fh, indent=1, sort_keys=True)


if __name__ == "__main__":
    main([int(a) for a in sys.argv[1:]] or [64, 65, 288, 512])
