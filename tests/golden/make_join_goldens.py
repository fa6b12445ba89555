"""Fixtures that pin the join side and the text reader to the reference's own code.

The reference's join has no test vectors of its own, so this script makes them by running
its code on seeded layers: oracle/_ref/gcmf_join_ref (built by
`make -C oracle REF_ROOT=<reference root>` from the reference's sources, see
oracle/ref/gcmf_join_ref_driver.cu) runs

  * the text reader ReadTextFormatPolygon2WithVector (SEQ_Overlay.h:285-390),
  * the CPU MBR join IntersectMBR_SEQ (SEQ_Overlay.h:510-565),
  * with --gpu, the GPU join stages of spatialJoin3.cu:226-318: the sort-based MBR sweep
    (GPU_MBR.h:339-539), Get_CMBR, Point_In_Polygon_Test, Count_CMF/Apply_CMF and
    Segment_Intersect_Join (GPU_Join.h).  These need a CUDA device.

    python tests/golden/make_join_goldens.py --out <dir> [--gpu]

writes <dir>/join_ref_<case>.npz per case and <dir>/reader_rules_ref.npz; the committed
copies live next to this script.  The layers are regenerated by the tests from the same
seeds (case_layers) and written with the engine's text writer; the fixtures carry the
SHA-256 of those files, so a test can check that it feeds the same bytes.

Every case stays inside the reference's fixed limits (see the driver's header):
coordinates in [1, 999], 8-64 vertices per polygon, at most 2,000 polygons per layer.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "gcmf-gh_b200"))
from gcmfgh import synth  # noqa: E402

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "gcmf_join_ref")
RULES_FILE = os.path.join(HERE, "reader_rules.txt")
CASES = ("small_join", "dense")


def _inside(layer, lo=1.0, hi=999.0):
    keep = [layer.ring(i) for i in range(layer.n_polys)
            if layer.ring(i).min() >= lo and layer.ring(i).max() <= hi]
    return synth.Layer.from_rings(keep)


def case_layers(name):
    """(base, overlay) of one case.
    small_join: the small-join workload (2,000 + 2,000 stars over [0, 1000]^2, 8-64
      vertices, radius log-normal(ln 5, 0.5), seed 0), less the polygons that leave
      [1, 999]^2.
    dense: 600 small stars (radius log-normal(ln 4, 0.6)) against 300 larger ones
      (log-normal(ln 12, 0.5)) over [100, 300]^2, seed 21: many containment candidates,
      contained pairs and edge-filter drops."""
    if name == "small_join":
        b, o = synth.small_join(0, 2000)
        return _inside(b), _inside(o)
    if name == "dense":
        rng = np.random.default_rng(21)
        nb, no = 600, 300
        b = synth.star_layer(rng, rng.integers(8, 65, size=nb), rng.uniform(100, 300, size=(nb, 2)),
                             rng.lognormal(np.log(4.0), 0.6, size=nb))
        o = synth.star_layer(rng, rng.integers(8, 65, size=no), rng.uniform(100, 300, size=(no, 2)),
                             rng.lognormal(np.log(12.0), 0.5, size=no))
        return _inside(b), _inside(o)
    raise ValueError(name)


def sha256(path):
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def write_case_text(name, d):
    """Writes the case's layers with the engine's text writer; returns the two paths."""
    import gcmfgh
    b, o = case_layers(name)
    pb, po = os.path.join(d, f"{name}_b.txt"), os.path.join(d, f"{name}_o.txt")
    gcmfgh.write_text_layer(pb, b)
    gcmfgh.write_text_layer(po, o)
    return pb, po


def _run(args, d):
    os.makedirs(d, exist_ok=True)
    subprocess.run([REF_BIN] + args + [d], check=True, stdout=subprocess.DEVNULL)


def _load(d, name, dtype):
    return np.fromfile(os.path.join(d, name + ".bin"), dtype=dtype)


def read_outputs(path, work):
    """The reference reader's arrays for one text file."""
    _run(["read", path], work)
    xy = _load(work, "layer_xy", np.float64)
    return {"vnum": _load(work, "layer_vnum", np.int32), "vps": _load(work, "layer_vps", np.int64),
            "key": _load(work, "layer_key", np.uint64), "mbr": _load(work, "layer_mbr", np.float64),
            "xy_sha": np.frombuffer(hashlib.sha256(xy.tobytes()).digest(), np.uint8), "xy": xy}


def make_case(name, out, gpu):
    with tempfile.TemporaryDirectory() as td:
        pb, po = write_case_text(name, td)
        rec = {"text_sha_b": np.array(sha256(pb)), "text_sha_o": np.array(sha256(po))}
        for side, p in (("b", pb), ("o", po)):
            r = read_outputs(p, os.path.join(td, "read_" + side))
            for k in ("vnum", "vps", "key", "mbr", "xy_sha"):
                rec[f"read_{side}_{k}"] = r[k]
        sd = os.path.join(td, "seq")
        _run(["seqjoin", pb, po], sd)
        rec["seq_b"] = _load(sd, "seq_b", np.int32)
        rec["seq_o"] = _load(sd, "seq_o", np.int32)
        if gpu:
            gd = os.path.join(td, "gpu")
            _run(["gpujoin", pb, po], gd)
            for k, dt in (("jxy", np.int32), ("cmbr", np.float64), ("pip_type", np.int8),
                          ("pip_candidate", np.int32), ("pip_flag", np.int32), ("join_flag", np.int32),
                          ("b_edge_ps", np.int64), ("o_edge_ps", np.int64), ("jxy2", np.int32),
                          ("b_edges", np.int16), ("o_edges", np.int16), ("seg_flag", np.int32),
                          ("counts", np.int64)):
                rec["gpu_" + k] = _load(gd, k, dt)
    np.savez_compressed(os.path.join(out, f"join_ref_{name}.npz"), **rec)
    return rec


def make_rules(out):
    with tempfile.TemporaryDirectory() as td:
        r = read_outputs(RULES_FILE, td)
    np.savez_compressed(os.path.join(out, "reader_rules_ref.npz"),
                        **{k: r[k] for k in ("vnum", "vps", "key", "mbr", "xy")})


def reference_join_by_pair(fx):
    """The reference GPU join's per-candidate arrays of a fixture, reordered from the
    sweep's emission order to ascending (base, overlay), as the engine and the oracle
    report them: b, o, cmbr (K,4), pip_type, pip_candidate, pip_flag, join_flag, bE, oE,
    seg_flag (0 for pairs the edge filter removed)."""
    jxy = fx["gpu_jxy"].reshape(-1, 2).astype(np.int64)
    K = jxy.shape[0]
    order = np.lexsort((jxy[:, 1], jxy[:, 0]))
    bps, ops = fx["gpu_b_edge_ps"], fx["gpu_o_edge_ps"]
    bE = np.diff(np.concatenate([[0], bps]))
    oE = np.diff(np.concatenate([[0], ops]))
    seg = np.zeros(K, np.int32)
    seg[fx["gpu_jxy2"]] = fx["gpu_seg_flag"]
    out = {"b": jxy[:, 0], "o": jxy[:, 1], "cmbr": fx["gpu_cmbr"].reshape(-1, 4), "pip_type": fx["gpu_pip_type"],
           "pip_candidate": fx["gpu_pip_candidate"], "pip_flag": fx["gpu_pip_flag"],
           "join_flag": fx["gpu_join_flag"], "bE": bE, "oE": oE, "seg_flag": seg}
    return {k: v[order] for k, v in out.items()}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--gpu", action="store_true", help="also run the reference's GPU join stages")
    a = ap.parse_args()
    if not os.path.exists(REF_BIN):
        sys.exit("oracle/_ref/gcmf_join_ref is missing: build it with make -C oracle REF_ROOT=<reference root>")
    os.makedirs(a.out, exist_ok=True)
    make_rules(a.out)
    for name in CASES:
        rec = make_case(name, a.out, a.gpu)
        msg = f"{name}: {len(rec['read_b_vnum'])} + {len(rec['read_o_vnum'])} polygons, {len(rec['seq_b'])} seq pairs"
        if a.gpu:
            c = rec["gpu_counts"]
            msg += (f"; gpu: {c[0]} candidates, {c[1]} containment candidates, {c[2]} within, "
                    f"{c[3]} after the edge filter, {c[5]} intersecting")
        print(msg, flush=True)


if __name__ == "__main__":
    main()
