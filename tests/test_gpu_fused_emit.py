"""The one-pass record count + emit (default) against the two-pass count, then emit: the
records land in another order, and every result must be the same bit for bit.  Covers
chunked and binned pairs, the exact predicates, and a clip that finds more records than
its arrays were sized for (the pass then runs again at the counted size)."""
import numpy as np
import pytest

import pyoracle
from gcmfgh import synth

pytestmark = pytest.mark.gpu

BIN_DEFAULT = 1 << 16


def _pairs_layers(pairs):
    base = synth.Layer.from_rings([p for p, _ in pairs])
    ovl = synth.Layer.from_rings([q for _, q in pairs])
    ids = np.arange(len(pairs), dtype=np.int32)
    return base, ovl, ids


def _clip(engine, base, ovl, pid, qid, fused, hint=0, bin_grid=BIN_DEFAULT, exact=False, union=False):
    import gcmfgh
    db, do = gcmfgh.DeviceLayer(base), gcmfgh.DeviceLayer(ovl)
    engine.set_tuning(fused_emit=fused, record_hint=hint, bin_grid=bin_grid)
    engine.set_precision(exact)
    engine.set_params(1e-7, 1e-7, union)
    try:
        info = engine.clip_batch(db, do, pid, qid)
        return info, engine.clip_result()
    finally:
        engine.set_tuning(fused_emit=1, record_hint=0, bin_grid=BIN_DEFAULT)
        engine.set_precision(False)
        engine.set_params(1e-7, 1e-7, False)


def _assert_same(a, b):
    assert np.array_equal(a.status, b.status)
    assert np.array_equal(a.count1, b.count1)
    assert np.array_equal(a.ncomp, b.ncomp)
    assert np.array_equal(a.comp_size, b.comp_size)
    assert np.array_equal(a.xy, b.xy)


@pytest.mark.parametrize("variant", [1, 2])
@pytest.mark.parametrize("exact", [False, True])
@pytest.mark.parametrize("union", [False, True])
def test_fused_matches_two_pass_and_oracle(engine, variant, exact, union):
    """variant 1: block-wide appends of the records; 2: one append per warp."""
    base, ovl, ids = _pairs_layers(synth.random_star_pairs(61, 800, 3, 90, spread=0.8))
    i2, r2 = _clip(engine, base, ovl, ids, ids, fused=0, exact=exact, union=union)
    i1, r1 = _clip(engine, base, ovl, ids, ids, fused=variant, exact=exact, union=union)
    assert i1["n_records"] == i2["n_records"] > 0
    _assert_same(r1, r2)
    o = pyoracle.clip_batch(base, ovl, ids, ids, union=union, exact=exact)
    assert np.array_equal(r1.status, o.status)
    assert np.array_equal(r1.xy, o.xy)
    assert np.array_equal(r1.comp_size, o.comp_size)


@pytest.mark.parametrize("variant", [1, 2])
@pytest.mark.parametrize("bin_grid", [0, 2000, BIN_DEFAULT])
@pytest.mark.parametrize("hint", [0, 1])
def test_fused_with_binned_pairs_and_overflow(engine, variant, bin_grid, hint):
    """bin_grid 0: every pair binned (its records after the chunked ones, of which there
    are none); 2000: a mix; hint 1: arrays of 4,097 records, far fewer than the clip
    finds, so the pass runs again at the counted size."""
    base, ovl, ids = _pairs_layers(synth.random_star_pairs(62, 600, 20, 300, spread=0.6))
    i2, r2 = _clip(engine, base, ovl, ids, ids, fused=0, bin_grid=bin_grid)
    i1, r1 = _clip(engine, base, ovl, ids, ids, fused=variant, hint=hint, bin_grid=bin_grid)
    assert i1["n_records"] == i2["n_records"]
    if hint:
        assert i1["n_records"] > 4097
    _assert_same(r1, r2)


def test_fused_join_clip_workload(engine):
    """A joined clip set (pairs of two star layers), fused with a stale hint from a
    smaller clip, then again with the hint this clip leaves behind."""
    import gcmfgh
    base, ovl = synth.small_join(5, 3000)
    db, do = gcmfgh.DeviceLayer(base), gcmfgh.DeviceLayer(ovl)
    engine.join(db, do)
    engine.set_tuning(fused_emit=0)
    try:
        ref_info = engine.clip_joined(db, do)
        ref = engine.clip_result()
    finally:
        engine.set_tuning(fused_emit=1)
    small_b, small_o, ids = _pairs_layers(synth.random_star_pairs(63, 4, 3, 8))
    engine.clip_batch(gcmfgh.DeviceLayer(small_b), gcmfgh.DeviceLayer(small_o), ids, ids)   # small hint
    engine.join(db, do)
    for _ in range(2):
        info = engine.clip_joined(db, do)
        assert info["n_records"] == ref_info["n_records"]
        _assert_same(engine.clip_result(), ref)
