"""Regenerates tests/golden/holed_pairs.npz: seeded multi-component pairs (star islands
with star holes, gcmfgh.synth.holed_pairs(5, 150)) and the output of the reference's own
sequential clipper on them (oracle/_ref/ghclip_ref "mbatch" mode, built from the
reference's GH-CUDA/lib sources), for intersection and for union.  Run after
`make -C oracle`, where the reference is mounted:

    python tests/golden/make_multi_goldens.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "gcmf-gh_b200"))

import pyoracle  # noqa: E402
from gcmfgh import synth  # noqa: E402


def pack_results(results, tag):
    ncomp = np.array([len(c) for c in results], np.int32)
    csz = np.array([len(x) for c in results for x in c], np.int32)
    xy = np.concatenate([x.reshape(-1) for c in results for x in c]) if csz.size else np.zeros(0)
    return {f"{tag}ncomp": ncomp, f"{tag}comp_size": csz, f"{tag}xy": xy}


def main():
    if not pyoracle.ref_available():
        raise SystemExit("build oracle/_ref first: make -C oracle")
    pairs = synth.holed_pairs(5, 150)
    out = {"kP": np.array([len(P) for P, _ in pairs], np.int32),
           "kQ": np.array([len(Q) for _, Q in pairs], np.int32),
           "sizes": np.array([len(r) for P, Q in pairs for r in P + Q], np.int32),
           "xy": np.concatenate([r.reshape(-1) for P, Q in pairs for r in P + Q])}
    out.update(pack_results(pyoracle.ref_clip_multi(pairs), "i_"))
    out.update(pack_results(pyoracle.ref_clip_multi(pairs, union=True), "u_"))
    np.savez_compressed(os.path.join(HERE, "holed_pairs.npz"), **out)
    print("wrote", os.path.join(HERE, "holed_pairs.npz"), len(pairs), "pairs")


if __name__ == "__main__":
    main()
