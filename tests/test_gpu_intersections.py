"""The intersection phase of one pair -- the reference's calculateIntersections
(gppolyclip_mDIV512.cu:1298-1640) -- through the C ABI (gh_calculate_intersections) and
through the C++ shim with the reference's signature, bit-exact against the oracle's
restatement (pinned to the reference's own merged lists in test_oracle.py): merged rings,
(int)(1e7 * alpha) keys, initial labels, 1-based neighbours, invalid flag and sizes."""
import os
import struct
import subprocess

import numpy as np
import pytest

import pyoracle
from conftest import GOLDEN, ROOT, load_poly
from gcmfgh import synth

pytestmark = pytest.mark.gpu


def _assert_same(got, exp):
    assert (got["n_p"], got["n_q"], got["invalid"]) == (exp["n_p"], exp["n_q"], exp["invalid"])
    if not exp["invalid"]:
        for f in pyoracle.INTERSECTION_FIELDS:
            assert np.array_equal(got[f], exp[f]), f


def _check_pairs(engine, pairs, exact=False):
    import gcmfgh
    lp = gcmfgh.DeviceLayer(synth.Layer.from_rings([P for P, _ in pairs]))
    lq = gcmfgh.DeviceLayer(synth.Layer.from_rings([Q for _, Q in pairs]))
    engine.set_precision(exact)
    try:
        for k, (P, Q) in enumerate(pairs):
            _assert_same(engine.calculate_intersections(lp, k, lq, k), pyoracle.pair_intersections(P, Q, exact=exact))
    finally:
        engine.set_precision(False)


def _ring_fixture_pairs():
    d = np.load(os.path.join(GOLDEN, "ring_pairs.npz"))
    op = oq = 0
    out = []
    for k in range(len(d["nP"])):
        out.append((d["P"][2 * op:2 * (op + d["nP"][k])].reshape(-1, 2),
                    d["Q"][2 * oq:2 * (oq + d["nQ"][k])].reshape(-1, 2)))
        op += d["nP"][k]
        oq += d["nQ"][k]
    return out


@pytest.mark.parametrize("exact", [False, True])
def test_fig_and_fixture_pairs(engine, exact):
    _check_pairs(engine, _ring_fixture_pairs(), exact)


@pytest.mark.parametrize("exact", [False, True])
def test_random_star_pairs(engine, exact):
    _check_pairs(engine, synth.random_star_pairs(11, 60, 20, 3000, spread=1.0), exact)


@pytest.mark.parametrize("exact", [False, True])
def test_degeneracy_classes(engine, exact):
    classes, pairs = synth.degeneracy_pairs(3, 400, vmax=400)
    pick = [p for c, p in zip(classes, pairs) if c != 0][:40] + pairs[:40]
    _check_pairs(engine, pick, exact)


def test_invalid_and_disjoint_pairs(engine):
    P, Q = synth.random_star_pairs(7, 1, 4, 12, spread=1.0)[0]
    sq = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], float)
    pairs = [(P * 1e-3, Q * 1e-3), (sq, sq + 5)]
    exp = [pyoracle.pair_intersections(a, b) for a, b in pairs]
    assert exp[0]["invalid"] == 1 and exp[1]["status"] == 2
    _check_pairs(engine, pairs)


def test_large_pair_binned_path(engine):
    """20,000 x 10,000 vertices: more edge pairs than the chunked path takes, so records
    come from the binned count/emit and the heavy-edge fills."""
    rng = np.random.default_rng(21)
    P = synth._star(rng, 20000, 0.0, 0.0, 1.0, 0.8, 1.2)
    Q = synth._star(rng, 10000, 0.05, 0.03, 1.0, 0.7, 1.3)
    _check_pairs(engine, [(P, Q)], exact=True)


def _read_shim_output(path):
    data = open(path, "rb").read()
    (n,) = struct.unpack_from("<q", data, 0)
    off = 8
    out = []
    for _ in range(n):
        n_p, n_q, inv = struct.unpack_from("<iii", data, off)
        off += 12
        r = {"n_p": n_p, "n_q": n_q, "invalid": inv}
        if not inv:
            for name, cnt, dt in (("xy_p", 2 * n_p, np.float64), ("xy_q", 2 * n_q, np.float64),
                                  ("alpha_p", n_p, np.int32), ("alpha_q", n_q, np.int32),
                                  ("label_p", n_p, np.int32), ("label_q", n_q, np.int32),
                                  ("neighbor_p", n_p, np.int32), ("neighbor_q", n_q, np.int32)):
                r[name] = np.frombuffer(data, dt, cnt, off).copy()
                off += cnt * np.dtype(dt).itemsize
        out.append(r)
    return out


def test_reference_signature_through_shims(tmp_path):
    """spatialJoin, then calculateIntersections with the reference's signature on the
    first 300 pairs of the clip set, as regularPolygonHandler calls it."""
    import gcmfgh
    base, ovl = synth.small_join(0, 2000)
    fb, fo, fr = tmp_path / "base.txt", tmp_path / "overlay.txt", tmp_path / "rings.bin"
    gcmfgh.write_text_layer(str(fb), base)
    gcmfgh.write_text_layer(str(fo), ovl)
    exe = tmp_path / "shim_intersections"
    lib = os.path.join(ROOT, "gcmf-gh_b200", "lib")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "shim_intersections.cpp"), "-o", str(exe), "-L", lib,
                    "-lgcmfgh_shims", f"-Wl,-rpath,{lib}"], check=True)
    env = dict(os.environ, GCMFGH_BASE_FILE=str(fb), GCMFGH_OVERLAY_FILE=str(fo))
    subprocess.run([str(exe), "1", "x", "300", str(fr)], check=True, env=env, timeout=300)
    got = _read_shim_output(fr)
    assert len(got) == 300
    rb, _ = gcmfgh.read_text_layer(str(fb))
    ro, _ = gcmfgh.read_text_layer(str(fo))
    j = pyoracle.join(rb, ro)
    sel = np.flatnonzero(j.clip == 1)[:300]
    for k, g in zip(sel, got):
        _assert_same(g, pyoracle.pair_intersections(rb.ring(int(j.b[k])), ro.ring(int(j.o[k]))))
