"""Exact-predicate mode of the oracle (CPU): its sign arithmetic against rational
arithmetic, its results on the reference's Fig goldens, and its behaviour on the
degeneracy classes of the precision workload."""
import os
from fractions import Fraction

import numpy as np
import pytest

import pyoracle
from conftest import GOLDEN, format_reference, load_poly
from gcmfgh import synth


def _near_collinear_rows(rng, n):
    p = rng.uniform(-1e3, 1e3, size=(n, 2))
    q = rng.uniform(-1e3, 1e3, size=(n, 2))
    t = rng.uniform(-0.5, 1.5, size=(n, 1))
    r = p + t * (q - p)
    steps = rng.integers(-3, 4, size=(n, 2))
    for k in range(n):                       # a few ulps off the line (or on it)
        for a in range(2):
            for _ in range(abs(int(steps[k, a]))):
                r[k, a] = np.nextafter(r[k, a], np.inf if steps[k, a] > 0 else -np.inf)
    return np.concatenate([p, q, r], axis=1)


def _sign(v):
    return (v > 0) - (v < 0)


def test_exact_orientation_signs_match_rational_arithmetic():
    rng = np.random.default_rng(11)
    rows = np.concatenate([_near_collinear_rows(rng, 3000), rng.uniform(-1, 1, size=(500, 6))])
    rows[:50, 4:6] = rows[:50, 0:2]          # coincident points
    got = pyoracle.exact_signs(rows)
    F = [[Fraction(float(v)) for v in row] for row in rows]
    want = [_sign((qx - px) * (ry - py) - (qy - py) * (rx - px)) for px, py, qx, qy, rx, ry in F]
    assert np.array_equal(got, np.array(want))
    # the FP64 expression gets a visible share of these wrong, so the test has teeth
    fp = np.sign((rows[:, 2] - rows[:, 0]) * (rows[:, 5] - rows[:, 1])
                 - (rows[:, 3] - rows[:, 1]) * (rows[:, 4] - rows[:, 0]))
    assert (fp != np.array(want)).sum() > 50


def test_exact_dot_signs_match_rational_arithmetic():
    rng = np.random.default_rng(12)
    base = _near_collinear_rows(rng, 2000)
    # (r - p) . (q - p) with r pushed towards the perpendicular through p
    d = base[:, 2:4] - base[:, 0:2]
    perp = np.stack([-d[:, 1], d[:, 0]], axis=1)
    r = base[:, 0:2] + perp * rng.uniform(0.5, 2.0, size=(2000, 1))
    rows = np.concatenate([r, base[:, 0:2], base[:, 2:4], base[:, 0:2]], axis=1)
    got = pyoracle.exact_signs(rows, dot=True)
    F = [[Fraction(float(v)) for v in row] for row in rows]
    want = [_sign((a - c) * (e - g) + (b - d_) * (f - h)) for a, b, c, d_, e, f, g, h in F]
    assert np.array_equal(got, np.array(want))


FIGS = ["Fig1", "Fig8", "Fig14", "Fig14cw", "Fig15", "Fig16", "Fig17", "Fig19"]


@pytest.mark.parametrize("name", FIGS)
@pytest.mark.parametrize("gpu_semantics", [False, True])
def test_exact_mode_reproduces_reference_figs(name, gpu_semantics):
    """The Figs' degeneracies are exact on their inputs, so exact predicates give the
    reference clipper's own output byte for byte."""
    f = lambda s: os.path.join(GOLDEN, "figs", f"{name}-{s}")
    P, Q = load_poly(f("P.poly"))[0], load_poly(f("Q.poly"))[0]
    r = pyoracle.clip_pair(P, Q, gpu_semantics=gpu_semantics, exact=True)
    assert r.status[0] == 0
    assert format_reference(r.components(0)) == open(f("R.run.poly")).read()


def _shoelace(c):
    x, y = c[:, 0], c[:, 1]
    return 0.5 * float(np.sum(x * np.roll(y, -1) - np.roll(x, -1) * y))


def test_exact_mode_degeneracy_classes():
    """No pair is invalid in exact mode; shared-vertex and collinear-overlap pairs (exact
    constructions) agree with the tolerance mode; 1e-12-translated copies keep the whole
    polygon as intersection and as union (|area| to 1e-9 relative)."""
    classes, pairs = synth.degeneracy_pairs(3, 1500, 4, 200)
    base = synth.Layer.from_rings([p for p, _ in pairs])
    ovl = synth.Layer.from_rings([q for _, q in pairs])
    ids = np.arange(len(pairs), dtype=np.int32)
    ex = pyoracle.clip_batch(base, ovl, ids, ids, exact=True)
    ref = pyoracle.clip_batch(base, ovl, ids, ids)
    assert set(np.unique(ex.status)) <= {0, 2}
    for c in (0, 1, 2):
        m = classes == c
        assert np.array_equal(ex.status[m], ref.status[m]) and np.array_equal(ex.count1[m], ref.count1[m])
        assert np.array_equal(ex.ncomp[m], ref.ncomp[m])
    exu = pyoracle.clip_batch(base, ovl, ids, ids, exact=True, union=True)
    for k in np.flatnonzero(classes == 3):
        aP = _shoelace(pairs[k][0])
        for res in (ex, exu):
            comps = res.components(k)
            assert len(comps) == 1
            assert abs(abs(_shoelace(comps[0])) - aP) <= 1e-9 * aP   # GH may trace either way
