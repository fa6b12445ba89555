"""Digests of the oracle's exact-mode results on the single-large-pair workload family
(star with nP vertices, radius U(0.8,1.2), centre (0,0) against a star with nQ vertices,
radius U(0.7,1.3), centre (0.05,0.03); seed 1), for bit-exact checks at sizes too large to
re-run the oracle inside a test.  Needs only the oracle library (make -C oracle):

    python tests/golden/make_large_pair_digests.py [nPxnQ ...]

Writes tests/golden/large_pair_digests.json: per size, status, P-side intersection count,
component count, vertex count and SHA-256 of the component sizes (int32 little-endian)
and of the vertices (float64 little-endian, x,y interleaved)."""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "gcmf-gh_b200"))

import pyoracle  # noqa: E402
from gcmfgh import synth  # noqa: E402

OUT = os.path.join(HERE, "large_pair_digests.json")


def digest(r):
    return {
        "status": int(r.status[0]), "count1": int(r.count1[0]), "ncomp": int(r.ncomp[0]),
        "nv": int(len(r.xy) // 2),
        "comp_size_sha256": hashlib.sha256(np.ascontiguousarray(r.comp_size, "<i4").tobytes()).hexdigest(),
        "xy_sha256": hashlib.sha256(np.ascontiguousarray(r.xy, "<f8").tobytes()).hexdigest(),
    }


def main(sizes):
    table = json.load(open(OUT)) if os.path.exists(OUT) else {}
    for nP, nQ in sizes:
        s, c = synth.large_pair(1, nP, nQ)
        one = np.array([0], np.int32)
        t = time.time()
        r = pyoracle.clip_batch(s, c, one, one, exact=True)
        d = digest(r)
        d["oracle_seconds"] = round(time.time() - t, 1)
        table[f"{nP}x{nQ}"] = d
        json.dump(table, open(OUT, "w"), indent=1, sort_keys=True)
        print(nP, nQ, d, flush=True)


if __name__ == "__main__":
    args = sys.argv[1:] or ["100000x50000", "200000x100000", "400000x200000", "1000000x500000"]
    main([tuple(int(v) for v in a.split("x")) for a in args])
