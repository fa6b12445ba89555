"""Regenerates the golden fixtures in tests/golden/ from the reference repository.

Run where the reference's sources are present, after
`make -C oracle REF_ROOT=<reference root>` has built oracle/_ref/ghclip_ref from them:

    GCMFGH_REFERENCE=<reference root> python tests/golden/make_goldens.py

Writes
  figs/<Name>-P.poly, figs/<Name>-Q.poly   the reference's GH test inputs
                                            (GH-CUDA/data, listed in GH-CUDA/ReadMe.txt:18-36)
  figs/<Name>-R.ref.poly                   the reference's published result where it has one
                                            (GH-CUDA/results/<Name>-R.poly)
  figs/<Name>-R.run.poly                   the output of the reference's own sequential
                                            clipper on the inputs, run here (oracle/_ref)
  synthetic_<n>.npz                        GH-CUDA/data/syntheticAlltoALL worst-case pairs
                                            ("count, then x,y per line") + reference output
  random_pairs.npz, random_pairs_union.npz seeded star pairs + reference output
"""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("GCMFGH_REFERENCE")
if not REF:
    sys.exit("set GCMFGH_REFERENCE to the directory that holds the reference's sources")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "gcmf-gh_b200"))

import pyoracle  # noqa: E402
from gcmfgh import synth  # noqa: E402

FIGS = [  # (name, P file, Q file, reference result file or None)
    ("Fig1", "Fig1-P.poly", "Fig1-Q.poly", "Fig1-R.poly"),
    ("Fig8", "Fig8-P.poly", "Fig8-Q.poly", None),            # its results file is empty
    ("Fig14", "Fig14-P.poly", "Fig14-Q.poly", "Fig14-R.poly"),
    ("Fig14cw", "Fig14-P-clockWise.poly", "Fig14-Q.poly", None),
    ("Fig15", "Fig15-P.poly", "Fig15-Q.poly", "Fig15-R.poly"),
    ("Fig16", "Fig16-P.poly", "Fig16-Q.poly", None),
    ("Fig17", "Fig17-P-Clockwise.poly", "Fig17-Q.poly", "Fig17-R.poly"),
    ("Fig18", "Fig18-P.poly", "Fig18-Q.poly", None),          # multi-component holes
    ("Fig19", "Fig19-P.poly", "Fig19-Q.poly", "Fig19-R.poly"),
]


def read_count_format(path):
    """'count' on the first line, then one 'x,y' per line."""
    with open(path) as f:
        n = int(f.readline())
        pts = [tuple(float(v) for v in f.readline().split(",")) for _ in range(n)]
    return np.array(pts, dtype=np.float64)


def pack(pairs, results):
    """npz arrays: pair vertex counts + coords, result components per pair."""
    np_, nq, xyp, xyq, ncomp, csz, rxy = [], [], [], [], [], [], []
    for (P, Q), comps in zip(pairs, results):
        np_.append(len(P)); nq.append(len(Q)); xyp.append(P.reshape(-1)); xyq.append(Q.reshape(-1))
        ncomp.append(len(comps))
        for c in comps:
            csz.append(len(c)); rxy.append(c.reshape(-1))
    cat = lambda a: np.concatenate(a) if a else np.zeros(0)
    return dict(nP=np.array(np_, np.int32), nQ=np.array(nq, np.int32), P=cat(xyp), Q=cat(xyq),
                ncomp=np.array(ncomp, np.int32), comp_size=np.array(csz, np.int32), xy=cat(rxy))


def main():
    if not pyoracle.ref_available():
        raise SystemExit("build oracle/_ref first: make -C oracle")
    figdir = os.path.join(HERE, "figs")
    os.makedirs(figdir, exist_ok=True)
    data = os.path.join(REF, "GH-CUDA", "data")
    res = os.path.join(REF, "GH-CUDA", "results")
    for name, pf, qf, rf in FIGS:
        for src, dst in ((pf, f"{name}-P.poly"), (qf, f"{name}-Q.poly")):
            with open(os.path.join(data, src)) as f, open(os.path.join(figdir, dst), "w") as g:
                g.write(f.read())
        if rf:
            with open(os.path.join(res, rf)) as f, open(os.path.join(figdir, f"{name}-R.ref.poly"), "w") as g:
                g.write(f.read())
        subprocess.run([pyoracle.REF_BIN, "text", os.path.join(figdir, f"{name}-P.poly"),
                        os.path.join(figdir, f"{name}-Q.poly"), os.path.join(figdir, f"{name}-R.run.poly")],
                       check=True, stdout=subprocess.DEVNULL)
    for n in (100,):
        d = os.path.join(data, "syntheticAlltoALL")
        P = read_count_format(os.path.join(d, f"worst-syntheticP_{n}.txt"))
        Q = read_count_format(os.path.join(d, f"worst-syntheticQ_{n}.txt"))
        out = pyoracle.ref_clip_pairs([(P, Q)])
        np.savez_compressed(os.path.join(HERE, f"synthetic_{n}.npz"), **pack([(P, Q)], out))
    pairs = synth.random_star_pairs(20240601, 400, 3, 40, spread=1.0)
    pairs = [pq for pq in pairs if _mbrs_overlap(*pq)]
    out = pyoracle.ref_clip_pairs(pairs)
    np.savez_compressed(os.path.join(HERE, "random_pairs.npz"), **pack(pairs, out))
    out = pyoracle.ref_clip_pairs(pairs, union=True)
    np.savez_compressed(os.path.join(HERE, "random_pairs_union.npz"), **pack(pairs, out))
    print("goldens written to", HERE)


def _mbrs_overlap(P, Q):
    return not (P[:, 0].min() > Q[:, 0].max() or P[:, 0].max() < Q[:, 0].min() or
                P[:, 1].min() > Q[:, 1].max() or P[:, 1].max() < Q[:, 1].min())


if __name__ == "__main__":
    main()
