"""GPU parity of the batched Greiner-Hormann clip against the oracle and the reference's
golden outputs.  Integer results (status, counts, component sizes) and every output
coordinate must be bit-identical: the kernels evaluate the reference's FP64 expressions
in the same order without FMA contraction, as the oracle does."""
import os

import numpy as np
import pytest

import pyoracle
from conftest import GOLDEN, format_reference, load_poly, same_components, unpack_pairs
from gcmfgh import synth

pytestmark = pytest.mark.gpu

FIGS = ["Fig1", "Fig8", "Fig14", "Fig14cw", "Fig15", "Fig16", "Fig17", "Fig19"]


def _device_layers(base, ovl):
    import gcmfgh
    return gcmfgh.DeviceLayer(base), gcmfgh.DeviceLayer(ovl)


def _assert_batch_equal(engine, base, ovl, pid, qid, union=False, eps_clean=1e-7):
    db, do = _device_layers(base, ovl)
    engine.set_params(1e-7, eps_clean, union)
    try:
        info = engine.clip_batch(db, do, pid, qid)
        r = engine.clip_result()
    finally:
        engine.set_params(1e-7, 1e-7, False)
    o = pyoracle.clip_batch(base, ovl, pid, qid, union=union, eps_clean=eps_clean)
    # error word 2 = a trace that did not close within its budget (status 3 pairs)
    assert engine.last_device_error() in ((0, 2) if (r.status == 3).any() else (0,))
    assert np.array_equal(r.status, o.status)
    assert np.array_equal(r.count1[r.status != 2], o.count1[o.status != 2])
    assert np.array_equal(r.ncomp, o.ncomp)
    assert np.array_equal(r.comp_size, o.comp_size)
    assert np.array_equal(r.xy, o.xy)
    return info, r


@pytest.mark.parametrize("name", FIGS)
def test_figs_equal_reference_output(engine, name):
    P = load_poly(os.path.join(GOLDEN, "figs", f"{name}-P.poly"))[0]
    Q = load_poly(os.path.join(GOLDEN, "figs", f"{name}-Q.poly"))[0]
    engine.clip_pair(P, Q)
    r = engine.clip_result()
    assert r.status[0] == 0
    assert format_reference(r.components(0)) == open(os.path.join(GOLDEN, "figs", f"{name}-R.run.poly")).read()


@pytest.mark.parametrize("fixture,union", [("random_pairs.npz", False), ("random_pairs_union.npz", True)])
def test_random_pairs_equal_reference_output(engine, fixture, union):
    pairs, expect = unpack_pairs(os.path.join(GOLDEN, fixture))
    engine.set_params(1e-7, 1e-7, union)
    try:
        for (P, Q), exp in list(zip(pairs, expect))[:120]:
            engine.clip_pair(P, Q)
            r = engine.clip_result()
            if r.status[0] == 0:
                assert same_components(r.components(0), exp)
    finally:
        engine.set_params(1e-7, 1e-7, False)


def test_all_to_all_comb_equals_reference(engine):
    (pair,), (exp,) = unpack_pairs(os.path.join(GOLDEN, "synthetic_100.npz"))
    engine.clip_pair(*pair)
    r = engine.clip_result()
    assert r.status[0] == 0 and len(exp) == 2500
    assert same_components(r.components(0), exp)


@pytest.mark.parametrize("seed", [5, 6])
@pytest.mark.parametrize("union", [False, True])
def test_batch_random_pairs_bit_exact(engine, seed, union):
    pairs = synth.random_star_pairs(seed, 2500, 3, 60, spread=1.0)
    base = synth.Layer.from_rings([p for p, _ in pairs])
    ovl = synth.Layer.from_rings([q for _, q in pairs])
    ids = np.arange(len(pairs), dtype=np.int32)
    info, r = _assert_batch_equal(engine, base, ovl, ids, ids, union=union)
    assert info["n_disjoint"] > 0 and (r.status == 0).sum() > 2000


def test_batch_cleanup_tolerance_of_merged_build(engine):
    """The merged GCMF-GH build cleans up with EPSILON 1e-12 (Constants.h:29)."""
    pairs = synth.random_star_pairs(9, 800, 3, 40, spread=0.6)
    base = synth.Layer.from_rings([p for p, _ in pairs])
    ovl = synth.Layer.from_rings([q for _, q in pairs])
    ids = np.arange(len(pairs), dtype=np.int32)
    _assert_batch_equal(engine, base, ovl, ids, ids, eps_clean=1e-12)


def _box(x1, y1, x2, y2):
    return np.array([[x1, y1], [x2, y1], [x2, y2], [x1, y2]], dtype=np.float64)


def degenerate_pairs():
    """Shared vertices, collinear overlapping edges, vertex-on-edge, identical and nested
    polygons, rotated and reflected copies: the special cases of polyclip.h:405-734."""
    sq = _box(0, 0, 4, 4)
    cases = [
        (sq, _box(2, 2, 6, 6)),                     # proper crossing
        (sq, _box(4, 0, 8, 4)),                     # shared edge, outside
        (sq, _box(0, 0, 2, 2)),                     # shared corner + collinear edges, inside
        (sq, _box(1, 1, 3, 3)),                     # nested
        (sq, sq.copy()),                            # identical
        (sq, sq[::-1].copy()),                      # identical, opposite orientation
        (sq, np.array([[2, 4], [6, 6], [6, 2]], float)),        # vertex on edge (T)
        (sq, np.array([[4, 4], [6, 6], [6, 2]], float)),        # vertex on vertex (V)
        (sq, np.array([[1, 4], [3, 4], [3, 7], [1, 7]], float)),   # overlapping edge segment
        (sq, np.array([[0, 2], [4, 2], [4, 3], [0, 3]], float)),   # strip across, shared sides
        (sq, np.array([[2, 0], [4, 2], [2, 4], [0, 2]], float)),   # diamond touching midpoints
        (np.array([[0, 0], [4, 0], [4, 4], [2, 2], [0, 4]], float),
         np.array([[2, 2], [3, 5], [1, 5]], float)),               # reflex vertex contact
        (sq, np.array([[-1, 1], [5, 1], [5, 3], [-1, 3]], float)),  # band through
    ]
    rng = np.random.default_rng(3)
    base_cases = list(cases)
    for P, Q in base_cases:                          # rotations of the start vertex
        for s in (1, 2):
            cases.append((np.roll(P, s, axis=0), np.roll(Q, -s, axis=0)))
    for P, Q in base_cases:                          # mirrored copies
        cases.append((P * np.array([-1.0, 1.0]), Q * np.array([-1.0, 1.0])))
    for _ in range(40):                              # shared exact vertex between random stars
        P, Q = synth.random_star_pairs(int(rng.integers(1 << 30)), 1, 4, 30, 0.5)[0]
        Q = Q.copy()
        Q[int(rng.integers(len(Q)))] = P[int(rng.integers(len(P)))]
        cases.append((P, Q))
    return cases


@pytest.mark.parametrize("union", [False, True])
def test_degenerate_cases_bit_exact(engine, union):
    cases = degenerate_pairs()
    base = synth.Layer.from_rings([p for p, _ in cases])
    ovl = synth.Layer.from_rings([q for _, q in cases])
    ids = np.arange(len(cases), dtype=np.int32)
    _assert_batch_equal(engine, base, ovl, ids, ids, union=union)


def test_degenerate_single_pair_entry_point(engine):
    """gh_clip_pair (P clipped against Q as given, no swap) equals the oracle."""
    for P, Q in degenerate_pairs()[:13]:
        engine.clip_pair(P, Q)
        r = engine.clip_result()
        o = pyoracle.clip_pair(P, Q, gpu_semantics=True)
        assert r.status[0] == o.status[0]
        if r.status[0] == 0:
            assert same_components(r.components(0), o.components(0))


def test_empty_and_disjoint_batches(engine):
    base = synth.Layer.from_rings([_box(0, 0, 1, 1)])
    ovl = synth.Layer.from_rings([_box(5, 5, 6, 6)])
    db, do = _device_layers(base, ovl)
    info = engine.clip_batch(db, do, np.zeros(0, np.int32), np.zeros(0, np.int32))
    assert info["n_pairs"] == 0 and info["n_vertices"] == 0
    info = engine.clip_batch(db, do, np.zeros(1, np.int32), np.zeros(1, np.int32))
    assert info["n_disjoint"] == 1 and info["n_components"] == 0


def test_medium_pair_bit_exact(engine):
    """A 20,000 x 10,000 vertex instance of the large-pair workload (star polygons around
    nearby centres): tens of thousands of intersections on one pair."""
    s, c = synth.large_pair(1, 20000, 10000)
    info, r = _assert_batch_equal(engine, s, c, np.array([0], np.int32), np.array([0], np.int32))
    assert r.count1[0] > 50000 and info["n_components"] > 10000
