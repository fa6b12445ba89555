"""The clip's alternative work distributions give the same results: binned edge search
(instead of enumerating a pair's edge grid) and grid-wide labelling/tracing (instead of
a warp per pair), forced on every pair and compared bit-exactly with the oracle; and a
large single pair on the default thresholds."""
import numpy as np
import pytest

import pyoracle
from gcmfgh import synth

pytestmark = pytest.mark.gpu

BIN_DEFAULT, BIG_DEFAULT, MID_DEFAULT, TILE_DEFAULT, WIDE_DEFAULT = 1 << 16, 1 << 18, 1 << 10, 96, 1 << 16


def _run(engine, base, ovl, pid, qid, union=False, bin_grid=BIN_DEFAULT, big_label=BIG_DEFAULT,
         mid_label=MID_DEFAULT, exact=False, tile_label=TILE_DEFAULT, wide_label=WIDE_DEFAULT):
    import gcmfgh
    db, do = gcmfgh.DeviceLayer(base), gcmfgh.DeviceLayer(ovl)
    engine.set_tuning(bin_grid=bin_grid, big_label=big_label, mid_label=mid_label, tile_label=tile_label,
                      wide_label=wide_label)
    engine.set_params(1e-7, 1e-7, union)
    engine.set_precision(exact)
    try:
        info = engine.clip_batch(db, do, pid, qid)
        r = engine.clip_result()
    finally:
        engine.set_tuning(bin_grid=BIN_DEFAULT, big_label=BIG_DEFAULT, mid_label=MID_DEFAULT,
                          tile_label=TILE_DEFAULT, wide_label=WIDE_DEFAULT)
        engine.set_params(1e-7, 1e-7, False)
        engine.set_precision(False)
    return info, r


def _assert_equal(r, o):
    assert np.array_equal(r.status, o.status)
    assert np.array_equal(r.count1[r.status != 2], o.count1[o.status != 2])
    assert np.array_equal(r.ncomp, o.ncomp)
    assert np.array_equal(r.comp_size, o.comp_size)
    assert np.array_equal(r.xy, o.xy)


def _pairs_layers(pairs):
    base = synth.Layer.from_rings([p for p, _ in pairs])
    ovl = synth.Layer.from_rings([q for _, q in pairs])
    ids = np.arange(len(pairs), dtype=np.int32)
    return base, ovl, ids


@pytest.mark.parametrize("union", [False, True])
def test_binned_search_every_pair(engine, union):
    base, ovl, ids = _pairs_layers(synth.random_star_pairs(21, 1500, 3, 80, spread=0.8))
    _, r = _run(engine, base, ovl, ids, ids, union=union, bin_grid=0)
    _assert_equal(r, pyoracle.clip_batch(base, ovl, ids, ids, union=union))


@pytest.mark.parametrize("union", [False, True])
def test_grid_labelling_every_pair(engine, union):
    base, ovl, ids = _pairs_layers(synth.random_star_pairs(22, 250, 3, 60, spread=0.8))
    _, r = _run(engine, base, ovl, ids, ids, union=union, big_label=0)
    _assert_equal(r, pyoracle.clip_batch(base, ovl, ids, ids, union=union))


@pytest.mark.parametrize("union", [False, True])
@pytest.mark.parametrize("exact", [False, True])
def test_block_labelling_every_pair(engine, union, exact):
    """Every pair labelled and traced by a whole thread block (persistent, work-stealing)."""
    base, ovl, ids = _pairs_layers(synth.random_star_pairs(23, 1200, 3, 120, spread=0.8))
    _, r = _run(engine, base, ovl, ids, ids, union=union, mid_label=0, exact=exact)
    _assert_equal(r, pyoracle.clip_batch(base, ovl, ids, ids, union=union, exact=exact))


@pytest.mark.parametrize("union", [False, True])
@pytest.mark.parametrize("exact", [False, True])
@pytest.mark.parametrize("tile_label", [0, 1 << 10])
@pytest.mark.parametrize("wide_label", [0, WIDE_DEFAULT])
def test_tile_and_warp_labelling_every_pair(engine, union, exact, tile_label, wide_label):
    """Every warp-sized pair labelled by one thread (tile_label 2^10), or by a whole warp
    with the one-thread path switched off (0); with the full-GPU register budget forced
    (wide_label 0) and with the per-pair-latency one this batch size gets by default."""
    base, ovl, ids = _pairs_layers(synth.random_star_pairs(24, 1500, 3, 90, spread=0.8))
    _, r = _run(engine, base, ovl, ids, ids, union=union, tile_label=tile_label, exact=exact,
                wide_label=wide_label)
    _assert_equal(r, pyoracle.clip_batch(base, ovl, ids, ids, union=union, exact=exact))


@pytest.mark.parametrize("wide_label", [0, WIDE_DEFAULT])
def test_tile_labelling_degenerate_cases(engine, wide_label):
    from test_gpu_clip import degenerate_pairs
    base, ovl, ids = _pairs_layers(degenerate_pairs())
    for union in (False, True):
        _, r = _run(engine, base, ovl, ids, ids, union=union, tile_label=1 << 10, wide_label=wide_label)
        _assert_equal(r, pyoracle.clip_batch(base, ovl, ids, ids, union=union))


def test_block_labelling_degenerate_cases(engine):
    from test_gpu_clip import degenerate_pairs
    base, ovl, ids = _pairs_layers(degenerate_pairs())
    for union in (False, True):
        _, r = _run(engine, base, ovl, ids, ids, union=union, mid_label=0)
        _assert_equal(r, pyoracle.clip_batch(base, ovl, ids, ids, union=union))


def test_block_labelling_medium_pair(engine):
    s, c = synth.large_pair(1, 20000, 10000)
    one = np.array([0], np.int32)
    _, r = _run(engine, s, c, one, one, mid_label=0)
    _assert_equal(r, pyoracle.clip_batch(s, c, one, one))


def test_grid_labelling_degenerate_cases(engine):
    from test_gpu_clip import degenerate_pairs
    base, ovl, ids = _pairs_layers(degenerate_pairs())
    for union in (False, True):
        _, r = _run(engine, base, ovl, ids, ids, union=union, big_label=0, bin_grid=0)
        _assert_equal(r, pyoracle.clip_batch(base, ovl, ids, ids, union=union))


def test_grid_paths_medium_pair(engine):
    s, c = synth.large_pair(1, 20000, 10000)
    one = np.array([0], np.int32)
    _, r = _run(engine, s, c, one, one, big_label=0)
    _assert_equal(r, pyoracle.clip_batch(s, c, one, one))


def test_large_pair_invalid_status_parity(engine):
    """A 50,000-vertex star against a 25,000-vertex star with the single-pair workload's
    radius distributions.  Under the absolute 1e-7 tolerance the near-radial spikes make
    P-side and Q-side intersection counts differ, so the pair is invalid; the status and
    the P-side count (455,748 edge pairs) must match the oracle exactly."""
    s, c = synth.large_pair(1, 50000, 25000)
    one = np.array([0], np.int32)
    info, r = _run(engine, s, c, one, one)
    assert info["n_error"] == 0
    o = pyoracle.clip_batch(s, c, one, one)
    _assert_equal(r, o)
    assert r.status[0] == 1 and r.count1[0] == 455748
