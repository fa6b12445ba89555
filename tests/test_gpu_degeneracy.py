"""The degeneracy-stressed batch at its real vertex counts (log-uniform on [4, 10,000]),
in both precision modes, against the oracle: every degenerate pair of a seeded batch plus
generic ones, and the pairs whose trace does not close.

In the reference's tolerance mode (eps 1e-7) a few pairs -- overlays translated by 1e-12
relative, whose every edge is an eps-overlap of the base's -- get labels that make the
trace walk endless.  The reference's own sequential clipper, run on these pairs, never
returns (its trace keeps appending vertices).  The engine and the oracle bound the walk
and report the pair as status 3 with no output; the exact mode clips them."""
import numpy as np
import pytest

import pyoracle
from gcmfgh import synth

pytestmark = pytest.mark.gpu

# pairs of degeneracy_pairs(seed 3, 2,000 pairs, [4, 10000]) whose tolerance-mode trace
# does not close (oracle status 3)
NON_CLOSING = [79, 1323, 1348, 1637, 1873]


def _clip(engine, base, ovl, ids, exact):
    import gcmfgh
    db, do = gcmfgh.DeviceLayer(base), gcmfgh.DeviceLayer(ovl)
    engine.set_precision(exact)
    try:
        info = engine.clip_batch(db, do, ids, ids)
        r = engine.clip_result()
    finally:
        engine.set_precision(False)
    return info, r


def _equal(r, o):
    assert np.array_equal(r.status, o.status)
    assert np.array_equal(r.ncomp, o.ncomp)
    assert np.array_equal(r.comp_size, o.comp_size)
    assert np.array_equal(r.xy, o.xy)


@pytest.fixture(scope="module")
def batch():
    classes, pairs = synth.degeneracy_pairs(5, 3000, 4, 10_000)
    rng = np.random.default_rng(0)
    deg = np.flatnonzero(classes > 0)
    gen = rng.choice(np.flatnonzero(classes == 0), size=150, replace=False)
    sel = np.sort(np.concatenate([deg, gen]))
    base = synth.Layer.from_rings([pairs[i][0] for i in sel])
    ovl = synth.Layer.from_rings([pairs[i][1] for i in sel])
    return classes[sel], base, ovl, np.arange(len(sel), dtype=np.int32)


@pytest.mark.parametrize("exact", [False, True])
def test_degeneracy_batch_full_vertex_counts(engine, batch, exact):
    classes, base, ovl, ids = batch
    assert (classes > 0).sum() > 100 and max(base.vnum.max(), ovl.vnum.max()) > 5000
    info, r = _clip(engine, base, ovl, ids, exact)
    o = pyoracle.clip_batch(base, ovl, ids, ids, exact=exact)
    _equal(r, o)
    assert info["n_error"] == int((o.status == 3).sum())


def test_non_closing_traces_reported_like_the_oracle(engine):
    _, pairs = synth.degeneracy_pairs(3, 2000, 4, 10_000)
    base = synth.Layer.from_rings([pairs[i][0] for i in NON_CLOSING])
    ovl = synth.Layer.from_rings([pairs[i][1] for i in NON_CLOSING])
    ids = np.arange(len(NON_CLOSING), dtype=np.int32)
    info, r = _clip(engine, base, ovl, ids, exact=False)
    o = pyoracle.clip_batch(base, ovl, ids, ids)
    assert list(o.status) == [3] * len(NON_CLOSING)
    _equal(r, o)
    assert info["n_error"] == len(NON_CLOSING)
    # the exact mode closes every one of them, as the oracle's exact mode does
    info, r = _clip(engine, base, ovl, ids, exact=True)
    o = pyoracle.clip_batch(base, ovl, ids, ids, exact=True)
    _equal(r, o)
    assert info["n_error"] == 0 and (o.status == 0).all()
