"""The engine's parallel GCMF text reader against the oracle's restatement of the
reference reader (SEQ_Overlay.h:285-390), and the writer's round trip."""
import os

import numpy as np
import pytest

import textformat
from gcmfgh import synth


@pytest.fixture(scope="module")
def gcmfgh_mod():
    import gcmfgh
    return gcmfgh


def test_round_trip_bit_exact(tmp_path, gcmfgh_mod):
    base, _ = synth.small_join(0, 500)
    p = tmp_path / "layer.txt"
    gcmfgh_mod.write_text_layer(str(p), base)
    for threads in (1, 3, 8):
        got, ids = gcmfgh_mod.read_text_layer(str(p), threads)
        assert np.array_equal(got.xy, base.xy) and np.array_equal(got.vnum, base.vnum)
        assert np.array_equal(ids, np.arange(base.n_polys))


def test_round_trip_extreme_magnitudes(tmp_path, gcmfgh_mod):
    rng = np.random.default_rng(5)
    rings = []
    for scale in (1e-9, 1e-3, 1.0, 1e4, 1e7, 1e12):
        r = rng.uniform(-1, 1, size=(6, 2)) * scale
        rings.append(r)
    layer = synth.Layer.from_rings(rings)
    p = tmp_path / "mag.txt"
    gcmfgh_mod.write_text_layer(str(p), layer)
    got, _ = gcmfgh_mod.read_text_layer(str(p))
    assert np.array_equal(got.xy, layer.xy)


def test_reader_matches_reference_rules(tmp_path, gcmfgh_mod):
    """Header skipped; MBR over header pairs and vertices; zero-width MBR polygons skipped
    (also when only the 12-fraction-digit keys coincide); trailing (0, 0) dropped; a last
    line without newline; odd token counts; separators other than spaces."""
    lines = [
        "some header 123\n",
        "7 0.0 0.0 2.0 2.0 0.0 0.0 2.0 0.0 2.0 2.0 0.0 2.0 0.0 0.0 \n",
        "8 1.0 1.0 1.0 3.0 1.0 1.0 1.0 2.0 1.0 3.0 1.0 1.0 \n",            # zero width: skipped
        "9 5.0000000000001 0 5.00000000000019 1 5.0000000000001 0 5.00000000000019 1 5.0000000000001 0\n",
        "10,-1.5,-1.5,-0.5,-0.5,(-1.5 -1.5),(-0.5 -1.5),(-0.5 -0.5),(-1.5 -1.5)\n",
        "\n",
        "11 3 3 4 4 3 3 4 3 4 4 3 3 7\n",                                   # odd count
        "12 10 10 12 12 10 10 12 10 12 12 10 10",                          # no final newline
    ]
    p = tmp_path / "rules.txt"
    p.write_text("".join(lines))
    want_xy, want_vnum, want_ids = textformat.read_text_layer(str(p))
    got, ids = gcmfgh_mod.read_text_layer(str(p))
    assert np.array_equal(ids, want_ids)
    assert np.array_equal(got.vnum, want_vnum)
    assert np.array_equal(got.xy, want_xy.reshape(-1))
    assert list(ids) == [7, 10, 11, 12]


def test_reader_matches_oracle_on_generated_layer(tmp_path, gcmfgh_mod):
    base, ovl = synth.small_join(0, 2000)
    for L, name in ((base, "b.txt"), (ovl, "o.txt")):
        p = tmp_path / name
        gcmfgh_mod.write_text_layer(str(p), L)
        want_xy, want_vnum, _ = textformat.read_text_layer(str(p))
        got, _ = gcmfgh_mod.read_text_layer(str(p), 4)
        assert np.array_equal(got.vnum, want_vnum) and np.array_equal(got.xy, want_xy.reshape(-1))
