"""Regenerates tests/golden/ring_pairs.npz: the reference's own merged vertex lists and
step-1 labels (oracle/_ref/ghclip_ref in "rings" mode, built from the reference's
GH-CUDA/lib sources) for the single-component Fig inputs and the first 120 seeded random
pairs of random_pairs.npz.  They pin the oracle's restatement of calculateIntersections
(gppolyclip_mDIV512.cu:1298-1640).  Run after `make -C oracle`, where the reference is
mounted:

    python tests/golden/make_ring_goldens.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import pyoracle  # noqa: E402
from conftest import load_poly, unpack_pairs  # noqa: E402

FIGS = ["Fig1", "Fig8", "Fig14", "Fig14cw", "Fig15", "Fig16", "Fig17", "Fig19"]


def main():
    if not pyoracle.ref_available():
        raise SystemExit("build oracle/_ref first: make -C oracle")
    pairs = [(load_poly(os.path.join(HERE, "figs", f"{n}-P.poly"))[0],
              load_poly(os.path.join(HERE, "figs", f"{n}-Q.poly"))[0]) for n in FIGS]
    rnd, _ = unpack_pairs(os.path.join(HERE, "random_pairs.npz"))
    pairs += rnd[:120]
    rings = pyoracle.ref_rings(pairs)
    out = {"nP": np.array([len(P) for P, _ in pairs], np.int32),
           "nQ": np.array([len(Q) for _, Q in pairs], np.int32),
           "P": np.concatenate([P.reshape(-1) for P, _ in pairs]),
           "Q": np.concatenate([Q.reshape(-1) for _, Q in pairs]),
           "lenP": np.array([len(r[0]["x"]) for r in rings], np.int32),
           "lenQ": np.array([len(r[1]["x"]) for r in rings], np.int32)}
    for side, tag in ((0, "p"), (1, "q")):
        for f in pyoracle.RING_FIELDS:
            out[f"{tag}_{f}"] = np.concatenate([r[side][f] for r in rings])
    np.savez_compressed(os.path.join(HERE, "ring_pairs.npz"), **out)
    print("wrote", os.path.join(HERE, "ring_pairs.npz"), len(pairs), "pairs")


if __name__ == "__main__":
    main()
