"""The join side and the text reader pinned to outputs of the reference's own code.

tests/golden/make_join_goldens.py ran, on seeded layers, the reference's text reader
(ReadTextFormatPolygon2WithVector, SEQ_Overlay.h:285-390), its CPU MBR join
(IntersectMBR_SEQ, SEQ_Overlay.h:510-565) and its GPU join stages (the sort-based MBR
sweep, Get_CMBR, Point_In_Polygon_Test, Count_CMF/Apply_CMF, Segment_Intersect_Join:
GPU_MBR.h / GPU_Join.h, in the order of spatialJoin3.cu:226-318), all built from the
reference's sources.  These tests hold the engine's text reader and the oracle's join to
those outputs; tests/test_gpu_join.py holds the engine's GPU join to the same fixtures.

Deviations that the inputs avoid by construction (each is documented with the engine):
the reference compares 12-fraction-digit decimal keys where the engine compares FP64
values, and its CPU join excludes touching MBRs; the fixtures' layers have no two MBR
coordinates that are equal, or equal to 12 fraction digits."""
import os

import numpy as np
import pytest

import pyoracle
import textformat
from conftest import GOLDEN
from golden import make_join_goldens as mjg

CASES = mjg.CASES


@pytest.fixture(scope="module")
def gcmfgh_mod():
    import gcmfgh
    return gcmfgh


@pytest.fixture(scope="module", params=CASES)
def case(request, tmp_path_factory, gcmfgh_mod):
    name = request.param
    fx = np.load(os.path.join(GOLDEN, f"join_ref_{name}.npz"))
    d = tmp_path_factory.mktemp(name)
    pb, po = mjg.write_case_text(name, str(d))
    # the same bytes the reference read
    assert mjg.sha256(pb) == str(fx["text_sha_b"]) and mjg.sha256(po) == str(fx["text_sha_o"])
    base, _ = gcmfgh_mod.read_text_layer(pb, 4)
    ovl, _ = gcmfgh_mod.read_text_layer(po, 4)
    return name, fx, base, ovl, pb, po


def _sha(a):
    import hashlib
    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest(), np.uint8)


def test_engine_reader_matches_reference_reader(case):
    _, fx, base, ovl, _, _ = case
    for side, L in (("b", base), ("o", ovl)):
        assert np.array_equal(L.vnum, fx[f"read_{side}_vnum"])
        assert np.array_equal(L.vps, fx[f"read_{side}_vps"])
        assert np.array_equal(_sha(L.xy), fx[f"read_{side}_xy_sha"])


def test_oracle_reader_keys_match_reference(case):
    """The restated CoordToMBR keys and atof MBRs equal the reference reader's."""
    _, fx, _, _, pb, po = case
    for side, p in (("b", pb), ("o", po)):
        _, vnum, _, keys, mbrs = textformat.read_text_layer(p, with_mbrs=True)
        assert np.array_equal(vnum, fx[f"read_{side}_vnum"])
        assert np.array_equal(keys.reshape(-1), fx[f"read_{side}_key"])
        assert np.array_equal(mbrs.reshape(-1), fx[f"read_{side}_mbr"])


def test_reader_rules_file(gcmfgh_mod):
    """Hand-written lines: header skipped, MBR over header pairs and vertices (polygon 14's
    header extends its MBR), zero-width MBR skipped, 12-digit key collision skipped,
    commas and parentheses as separators, an odd token count, no final newline."""
    fx = np.load(os.path.join(GOLDEN, "reader_rules_ref.npz"))
    path = os.path.join(GOLDEN, "reader_rules.txt")
    got, ids = gcmfgh_mod.read_text_layer(path)
    assert np.array_equal(got.vnum, fx["vnum"]) and np.array_equal(got.vps, fx["vps"])
    assert np.array_equal(got.xy, fx["xy"])
    assert list(ids) == [7, 10, 11, 13, 14, 12]
    xy, vnum, _, keys, mbrs = textformat.read_text_layer(path, with_mbrs=True)
    assert np.array_equal(xy.reshape(-1), fx["xy"]) and np.array_equal(vnum, fx["vnum"])
    assert np.array_equal(keys.reshape(-1), fx["key"]) and np.array_equal(mbrs.reshape(-1), fx["mbr"])


def test_oracle_candidates_match_reference_cpu_join(case):
    _, fx, base, ovl, _, _ = case
    o = pyoracle.join(base, ovl)
    ref = sorted(zip(fx["seq_b"].tolist(), fx["seq_o"].tolist()))
    assert list(zip(o.b.tolist(), o.o.tolist())) == ref


def test_no_ties_in_fixture_layers(case):
    """The layers avoid the documented deviations: no MBR x (or y) coordinate of one layer
    equals one of the other layer, so strict, closed, key and FP64 tests all agree."""
    _, fx, _, _, _, _ = case
    for a, b in ((0, 0), (0, 2), (2, 0), (2, 2), (1, 1), (1, 3), (3, 1), (3, 3)):
        kb = fx["read_b_key"].reshape(-1, 4)[:, a]
        ko = fx["read_o_key"].reshape(-1, 4)[:, b]
        assert np.intersect1d(kb, ko).size == 0


def test_oracle_join_stages_match_reference_gpu_join(case):
    """Candidates, common MBRs, containment candidates and results, the edge filter's
    per-pair edge counts and drops, and the segment refine, pair by pair."""
    name, fx, base, ovl, _, _ = case
    if "gpu_jxy" not in fx.files:
        pytest.skip("fixture made without the reference's GPU stages")
    r = mjg.reference_join_by_pair(fx)
    o = pyoracle.join(base, ovl)
    assert np.array_equal(o.b, r["b"]) and np.array_equal(o.o, r["o"])
    assert np.array_equal(o.cmbr, r["cmbr"])
    assert np.array_equal(o.pip_type, r["pip_type"])
    assert np.array_equal(o.pip_type > 0, r["pip_candidate"] > 0)
    assert np.array_equal(o.pip_flag, r["pip_flag"])
    assert np.array_equal(o.join_flag, r["join_flag"])
    assert np.array_equal(o.bE, r["bE"]) and np.array_equal(o.oE, r["oE"])
    assert np.array_equal(o.seg_flag, r["seg_flag"])
    c = fx["gpu_counts"]
    assert c[0] == len(o.b) and c[1] == int((o.pip_type > 0).sum()) and c[2] == int(o.pip_flag.sum())
    assert c[3] == int(o.join_flag.sum()) and c[5] == int(o.seg_flag.sum())
    # the cases exercise every stage
    assert c[1] > 0 and c[3] > 0 and c[5] > 0
    if name == "dense":
        assert c[2] > 0 and int(((o.join_flag == 0) & (o.pip_flag == 0)).sum()) > 0
