"""Exact-predicate mode on the GPU, bit-exact against the oracle's exact mode: random
pairs, the special-case set, the degeneracy classes of the precision workload (shared
vertices, collinear overlaps, 1e-12 translations), the binned and grid-wide paths, and
a 20,000 x 10,000-vertex pair."""
import numpy as np
import pytest

import pyoracle
from gcmfgh import synth

pytestmark = pytest.mark.gpu

BIN_DEFAULT, BIG_DEFAULT = 1 << 16, 1 << 18


def _run(engine, base, ovl, ids_p, ids_q, union=False, bin_grid=BIN_DEFAULT, big_label=BIG_DEFAULT):
    import gcmfgh
    db, do = gcmfgh.DeviceLayer(base), gcmfgh.DeviceLayer(ovl)
    engine.set_tuning(bin_grid=bin_grid, big_label=big_label)
    engine.set_params(1e-7, 1e-7, union)
    engine.set_precision(True)
    try:
        info = engine.clip_batch(db, do, ids_p, ids_q)
        r = engine.clip_result()
    finally:
        engine.set_precision(False)
        engine.set_tuning(bin_grid=BIN_DEFAULT, big_label=BIG_DEFAULT)
        engine.set_params(1e-7, 1e-7, False)
    assert info["n_error"] == 0
    return r


def _assert_equal(r, o):
    assert np.array_equal(r.status, o.status)
    assert np.array_equal(r.count1[r.status != 2], o.count1[o.status != 2])
    assert np.array_equal(r.ncomp, o.ncomp)
    assert np.array_equal(r.comp_size, o.comp_size)
    assert np.array_equal(r.xy, o.xy)


def _layers(pairs):
    base = synth.Layer.from_rings([p for p, _ in pairs])
    ovl = synth.Layer.from_rings([q for _, q in pairs])
    return base, ovl, np.arange(len(pairs), dtype=np.int32)


@pytest.mark.parametrize("union", [False, True])
def test_exact_random_pairs(engine, union):
    base, ovl, ids = _layers(synth.random_star_pairs(31, 3000, 3, 60, spread=0.8))
    r = _run(engine, base, ovl, ids, ids, union=union)
    _assert_equal(r, pyoracle.clip_batch(base, ovl, ids, ids, union=union, exact=True))


@pytest.mark.parametrize("union", [False, True])
def test_exact_special_cases(engine, union):
    from test_gpu_clip import degenerate_pairs
    base, ovl, ids = _layers(degenerate_pairs())
    r = _run(engine, base, ovl, ids, ids, union=union)
    _assert_equal(r, pyoracle.clip_batch(base, ovl, ids, ids, union=union, exact=True))


@pytest.mark.parametrize("union", [False, True])
def test_exact_degeneracy_classes(engine, union):
    classes, pairs = synth.degeneracy_pairs(3, 3000, 4, 300)
    base, ovl, ids = _layers(pairs)
    r = _run(engine, base, ovl, ids, ids, union=union)
    o = pyoracle.clip_batch(base, ovl, ids, ids, union=union, exact=True)
    _assert_equal(r, o)
    assert set(np.unique(r.status)) <= {0, 2}
    assert (classes == 3).sum() > 0 and (classes == 2).sum() > 0 and (classes == 1).sum() > 0


def test_exact_binned_and_grid_paths(engine):
    classes, pairs = synth.degeneracy_pairs(33, 600, 4, 120)
    base, ovl, ids = _layers(pairs)
    o = pyoracle.clip_batch(base, ovl, ids, ids, exact=True)
    _assert_equal(_run(engine, base, ovl, ids, ids, bin_grid=0), o)
    _assert_equal(_run(engine, base, ovl, ids, ids, big_label=0), o)


def test_exact_medium_pair(engine):
    s, c = synth.large_pair(1, 20000, 10000)
    one = np.array([0], np.int32)
    r = _run(engine, s, c, one, one)
    o = pyoracle.clip_batch(s, c, one, one, exact=True)
    _assert_equal(r, o)
    assert r.status[0] == 0 and r.count1[0] == 72912
