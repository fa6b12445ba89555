"""CPU tests of the oracle: pinned to the reference's golden vectors and to the output of
the reference's own sequential clipper (fixtures made by tests/golden/make_goldens.py)."""
import os

import numpy as np
import pytest

import pyoracle
from conftest import GOLDEN, format_reference, load_poly, same_components, unpack_pairs
from gcmfgh import synth

# Fig18 has several components per input (a polygon with holes); the join-and-clip path
# clips single-component layer polygons (GH-CUDA/ghcuda.cpp:64-91 takes one polygon per
# side), so it is not among the single-pair golden cases.
FIGS = ["Fig1", "Fig8", "Fig14", "Fig14cw", "Fig15", "Fig16", "Fig17", "Fig19"]


def _fig(name, suffix):
    return os.path.join(GOLDEN, "figs", f"{name}-{suffix}")


@pytest.mark.parametrize("name", FIGS)
@pytest.mark.parametrize("gpu_semantics", [False, True])
def test_oracle_reproduces_reference_clipper_on_figs(name, gpu_semantics):
    P = load_poly(_fig(name, "P.poly"))[0]
    Q = load_poly(_fig(name, "Q.poly"))[0]
    r = pyoracle.clip_pair(P, Q, gpu_semantics=gpu_semantics)
    assert r.status[0] == 0
    assert format_reference(r.components(0)) == open(_fig(name, "R.run.poly")).read()


@pytest.mark.parametrize("name", ["Fig1", "Fig14", "Fig15", "Fig19"])
def test_reference_published_results_byte_identical(name):
    """The reference's published results equal its own clipper run here (pins oracle/_ref)."""
    assert open(_fig(name, "R.ref.poly")).read() == open(_fig(name, "R.run.poly")).read()


def test_fig17_published_result_component_count():
    ref = load_poly(_fig("Fig17", "R.ref.poly"))
    run = load_poly(_fig("Fig17", "R.run.poly"))
    assert len(ref) == len(run) == 116
    canon = lambda cs: sorted(sorted(map(tuple, np.round(c, 3))) for c in cs)
    assert canon(ref) == canon(run)


@pytest.mark.parametrize("fixture,union", [("random_pairs.npz", False), ("random_pairs_union.npz", True)])
def test_oracle_matches_reference_clipper_random(fixture, union):
    pairs, expect = unpack_pairs(os.path.join(GOLDEN, fixture))
    assert len(pairs) > 300
    for (P, Q), exp in zip(pairs, expect):
        cpu = pyoracle.clip_pair(P, Q, union=union, gpu_semantics=False)
        assert same_components(cpu.components(0), exp)
        gpu = pyoracle.clip_pair(P, Q, union=union, gpu_semantics=True)
        if gpu.status[0] == 0:
            assert same_components(gpu.components(0), exp)


def test_oracle_matches_reference_on_all_to_all_comb():
    (pair,), (exp,) = unpack_pairs(os.path.join(GOLDEN, "synthetic_100.npz"))
    r = pyoracle.clip_pair(*pair, gpu_semantics=True)
    assert r.status[0] == 0
    assert len(exp) == 2500
    assert same_components(r.components(0), exp)


def test_eps_clean_changes_only_cleanup():
    P, Q = synth.random_star_pairs(7, 1, 30, 30, 0.2)[0]
    a = pyoracle.clip_pair(P, Q, eps_clean=1e-7)
    b = pyoracle.clip_pair(P, Q, eps_clean=1e-12)
    assert a.count1[0] == b.count1[0]


# ------------------------------------------------------------------ join oracle

def test_join_decomposition_equals_bruteforce_small_config():
    b, o = synth.small_join()
    r = pyoracle.join(b, o)
    bb, oo = pyoracle.join_bruteforce(b, o)
    assert len(r.b) == 1813
    assert np.array_equal(r.b, bb) and np.array_equal(r.o, oo)
    assert r.clip.sum() == r.pip_flag.sum() + r.seg_flag.sum()


def _box(x1, y1, x2, y2):
    return np.array([[x1, y1], [x2, y1], [x2, y2], [x1, y2]], dtype=np.float64)


def test_sweep_tie_rule_on_touching_mbrs():
    """Overlay starting exactly where a base ends is rejected; the mirror case (base
    starting where an overlay ends), corner and y touches are accepted
    (GPU_MBR.h:339-415 over a stable sort that puts base endpoints first)."""
    base = synth.Layer.from_rings([_box(0, 0, 1, 1)])
    ovl = synth.Layer.from_rings([
        _box(1, 0, 2, 1),      # x1o == x2b          -> rejected
        _box(-1, 0, 0, 1),     # x2o == x1b          -> accepted
        _box(0, 1, 1, 2),      # y touch             -> accepted
        _box(0.5, 0.5, 3, 3),  # proper overlap      -> accepted
        _box(1, 1, 2, 2),      # corner, x1o == x2b  -> rejected
        _box(5, 5, 6, 6),      # disjoint            -> rejected
    ])
    r = pyoracle.join(base, ovl)
    assert list(zip(r.b, r.o)) == [(0, 1), (0, 2), (0, 3)]
    bb, oo = pyoracle.join_bruteforce(base, ovl)
    assert list(zip(bb, oo)) == [(0, 1), (0, 2), (0, 3)]


def test_zero_width_mbr_never_joins():
    base = synth.Layer.from_rings([np.array([[0, 0], [0, 1], [0, 2]], float), _box(0, 0, 1, 1)])
    ovl = synth.Layer.from_rings([_box(-1, -1, 3, 3)])
    r = pyoracle.join(base, ovl)
    assert list(r.valid_b) == [0, 1]
    assert list(zip(r.b, r.o)) == [(1, 0)]
    assert r.pip_type[0] == 1 and r.pip_flag[0] == 1 and r.clip[0] == 1


def test_containment_and_disjoint_boundaries():
    base = synth.Layer.from_rings([_box(0, 0, 10, 10), _box(20, 20, 30, 30)])
    ovl = synth.Layer.from_rings([_box(2, 2, 3, 3), _box(25, 15, 35, 25)])
    r = pyoracle.join(base, ovl)
    pairs = list(zip(r.b, r.o))
    assert pairs == [(0, 0), (1, 1)]
    assert r.pip_type[0] == 2 and r.pip_flag[0] == 1        # base contains overlay
    assert r.pip_flag[1] == 0 and r.seg_flag[1] == 1         # crossing boundaries
    res = pyoracle.clip_batch(base, ovl, r.b, r.o)
    assert list(res.ncomp) == [1, 1]
    assert same_components(res.components(0), [_box(2, 2, 3, 3)])
