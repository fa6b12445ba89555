"""Multi-component pairs (outer rings and holes) through gh_clip_multi, bit-exact against
the oracle's restatement of the reference's component loops (which reproduces the
reference's own clipper on Fig18, Fig19 and the seeded holed pairs, test_oracle.py)."""
import os

import numpy as np
import pytest

import pyoracle
from conftest import GOLDEN, format_reference, load_poly, same_components, unpack_multi
from gcmfgh import synth

pytestmark = pytest.mark.gpu


def _gpu(engine, P, Q, union=False, exact=False):
    engine.set_params(1e-7, 1e-7, union)
    engine.set_precision(exact)
    try:
        info = engine.clip_multi(P, Q)
        r = engine.clip_result()
    finally:
        engine.set_precision(False)
        engine.set_params(1e-7, 1e-7, False)
    assert info["n_pairs"] == 1
    return r


@pytest.mark.parametrize("name", ["Fig18", "Fig19", "Fig1", "Fig17"])
def test_figs_all_components(engine, name):
    P = load_poly(os.path.join(GOLDEN, "figs", f"{name}-P.poly"))
    Q = load_poly(os.path.join(GOLDEN, "figs", f"{name}-Q.poly"))
    r = _gpu(engine, P, Q)
    assert r.status[0] == 0
    assert format_reference(r.components(0)) == open(os.path.join(GOLDEN, "figs", f"{name}-R.run.poly")).read()


@pytest.mark.parametrize("union", [False, True])
def test_holed_pairs_match_reference(engine, union):
    pairs, inter, uni = unpack_multi(os.path.join(GOLDEN, "holed_pairs.npz"))
    for (P, Q), exp in zip(pairs, uni if union else inter):
        r = _gpu(engine, P, Q, union=union)
        assert r.status[0] == 0
        assert same_components(r.components(0), exp)


@pytest.mark.parametrize("exact", [False, True])
def test_holed_pairs_against_oracle(engine, exact):
    for P, Q in synth.holed_pairs(17, 60, 20, 400):
        r = _gpu(engine, P, Q, exact=exact)
        o = pyoracle.clip_multi(P, Q, exact=exact)
        assert r.status[0] == o.status[0]
        assert r.count1[0] == o.count1[0]
        assert same_components(r.components(0), o.components(0))


def test_single_rings_equal_single_pair(engine):
    for P, Q in synth.random_star_pairs(11, 40, 20, 500):
        r = _gpu(engine, [P], [Q])
        o = pyoracle.clip_pair(P, Q)
        assert r.status[0] == o.status[0]
        if o.status[0] == 0:
            assert same_components(r.components(0), o.components(0))


def test_invalid_ring_pair_makes_pair_invalid(engine):
    P, Q = synth.random_star_pairs(7, 1, 4, 12, spread=1.0)[0]
    hole = synth._star(np.random.default_rng(1), 8, 0.0, 0.0, 0.1, 0.5, 1.0)
    r = _gpu(engine, [P * 1e-3, hole * 50], [Q * 1e-3])
    o = pyoracle.clip_multi([P * 1e-3, hole * 50], [Q * 1e-3])
    assert o.status[0] == 1 and r.status[0] == 1 and r.ncomp[0] == 0


def test_large_island_with_many_holes(engine):
    """A 6,000-vertex island with 24 holes against a 4,000-vertex island with 16 holes."""
    rng = np.random.default_rng(23)

    def island(cx, n, holes):
        rings = [synth._star(rng, n, cx, 0.0, 10.0, 0.8, 1.0)]
        for t in range(holes):
            ang = 2 * np.pi * t / holes
            rings.append(synth._star(rng, 40, cx + 5 * np.cos(ang), 5 * np.sin(ang), 0.6, 0.5, 1.0))
        return rings

    P, Q = island(0.0, 6000, 24), island(3.0, 4000, 16)
    for exact in (False, True):
        r = _gpu(engine, P, Q, exact=exact)
        o = pyoracle.clip_multi(P, Q, exact=exact)
        assert r.status[0] == o.status[0] == 0
        assert len(o.components(0)) > 5
        assert same_components(r.components(0), o.components(0))


def _gpu_batch(engine, pairs, union=False, exact=False):
    engine.set_params(1e-7, 1e-7, union)
    engine.set_precision(exact)
    try:
        info = engine.clip_multi_batch(pairs)
        r = engine.clip_result()
    finally:
        engine.set_precision(False)
        engine.set_params(1e-7, 1e-7, False)
    assert info["n_pairs"] == len(pairs)
    return r


@pytest.mark.parametrize("union", [False, True])
def test_batch_of_holed_pairs_matches_reference(engine, union):
    """The reference clipper's results for every holed pair, from one batched call."""
    pairs, inter, uni = unpack_multi(os.path.join(GOLDEN, "holed_pairs.npz"))
    r = _gpu_batch(engine, pairs, union=union)
    for i, exp in enumerate(uni if union else inter):
        assert r.status[i] == 0
        assert same_components(r.components(i), exp)


@pytest.mark.parametrize("exact", [False, True])
def test_batch_equals_single_calls_and_oracle(engine, exact):
    """A mixed batch (holed pairs, single rings, one invalid pair, the figures): each pair's
    result equals its own gh_clip_multi call bit for bit, and the oracle's."""
    pairs = [(P, Q) for P, Q in synth.holed_pairs(31, 40, 20, 300)]
    pairs += [([P], [Q]) for P, Q in synth.random_star_pairs(32, 20, 5, 200)]
    P, Q = synth.random_star_pairs(7, 1, 4, 12, spread=1.0)[0]
    hole = synth._star(np.random.default_rng(1), 8, 0.0, 0.0, 0.1, 0.5, 1.0)
    pairs.append(([P * 1e-3, hole * 50], [Q * 1e-3]))
    for name in ("Fig18", "Fig19"):
        pairs.append((load_poly(os.path.join(GOLDEN, "figs", f"{name}-P.poly")),
                      load_poly(os.path.join(GOLDEN, "figs", f"{name}-Q.poly"))))
    r = _gpu_batch(engine, pairs, exact=exact)
    if not exact:                      # the tolerance classification disagrees on P and Q sides
        assert r.status[len(pairs) - 3] == 1
    for i, (P, Q) in enumerate(pairs):
        s = _gpu(engine, P, Q, exact=exact)
        assert r.status[i] == s.status[0]
        assert r.count1[i] == s.count1[0]
        assert r.ncomp[i] == s.ncomp[0]
        a, b = r.components(i), s.components(0)
        assert len(a) == len(b) and all(np.array_equal(x, y) for x, y in zip(a, b))
        o = pyoracle.clip_multi(P, Q, exact=exact)
        assert r.status[i] == o.status[0]
        if o.status[0] == 0:
            assert same_components(a, o.components(0))
