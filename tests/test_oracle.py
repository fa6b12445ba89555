"""CPU tests of the oracle: pinned to the reference's golden vectors and to the output of
the reference's own sequential clipper (fixtures made by tests/golden/make_goldens.py)."""
import os

import numpy as np
import pytest

import pyoracle
from conftest import GOLDEN, format_reference, load_poly, same_components, unpack_pairs
from gcmfgh import synth

# Single-pair cases take the first component of each input, as the join-and-clip path
# does (GH-CUDA/ghcuda.cpp:64-91 takes one polygon per side).  Fig18 (holes) and all of
# Fig19's components are the multi-component cases further down.
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


def _ring_pairs():
    d = np.load(os.path.join(GOLDEN, "ring_pairs.npz"))
    op = oq = lp = lq = 0
    for k in range(len(d["nP"])):
        P = d["P"][2 * op:2 * (op + d["nP"][k])].reshape(-1, 2)
        Q = d["Q"][2 * oq:2 * (oq + d["nQ"][k])].reshape(-1, 2)
        ref = ({f: d[f"p_{f}"][lp:lp + d["lenP"][k]] for f in pyoracle.RING_FIELDS},
               {f: d[f"q_{f}"][lq:lq + d["lenQ"][k]] for f in pyoracle.RING_FIELDS})
        op += d["nP"][k]; oq += d["nQ"][k]; lp += d["lenP"][k]; lq += d["lenQ"][k]
        yield P, Q, ref


def test_pair_intersections_match_reference_lists():
    """The oracle's calculateIntersections outputs against the reference's own merged lists
    (computeIntersections + step-1 labels of GH-CUDA/lib/polyclip.h, fixture made by
    tests/golden/make_ring_goldens.py): same vertices in the same order, same links, the
    inserted vertices' keys equal (int)(1e7 * alpha), same initial labels.  Labels are
    compared where the GPU's rule for 'linked neighbour' (key != -100,
    gppolyclip_mDIV512.cu:1190-1201) agrees with the list's intersection flag: the source
    vertex of an X-overlap (type 5) is linked but keeps the key -100 on the GPU."""
    n = 0
    for P, Q, ref in _ring_pairs():
        r = pyoracle.pair_intersections(P, Q)
        assert r["status"] == 0
        quirkP = (r["neighbor_p"] != 0) & (r["alpha_p"] == -100)
        for tag, R in (("p", ref[0]), ("q", ref[1])):
            assert r["n_" + tag] == len(R["x"])
            xy = r["xy_" + tag].reshape(-1, 2)
            assert np.array_equal(xy[:, 0], R["x"]) and np.array_equal(xy[:, 1], R["y"])
            nb = r["neighbor_" + tag]
            assert np.array_equal(nb != 0, R["inter"] == 1)
            m = R["inter"] == 1
            assert np.array_equal(nb[m] - 1, R["nb"][m])
            ins = R["source"] == 0
            assert np.array_equal(r["alpha_" + tag][ins], (1e7 * R["alpha"][ins]).astype(np.int64))
        lbP = r["label_p"]
        npv = len(lbP)
        keyed = np.flatnonzero(lbP != -100)
        clean = keyed[~(quirkP[(keyed - 1) % npv] | quirkP[(keyed + 1) % npv])]
        got = np.where(lbP[clean] == -102, 0, lbP[clean])
        assert np.array_equal(got, ref[0]["label"][clean])
        qn = r["neighbor_p"][clean] - 1
        assert np.array_equal(np.where(r["label_q"][qn] == -102, 0, r["label_q"][qn]), ref[1]["label"][qn])
        n += 1
    assert n == 128


def test_pair_intersections_invalid_and_disjoint():
    # disjoint MBRs: the rings come back unchanged, every vertex plain
    P = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], float)
    r = pyoracle.pair_intersections(P, P + 5)
    assert r["status"] == 2 and r["n_p"] == 4 and r["n_q"] == 4
    assert np.array_equal(r["xy_p"], P.reshape(-1)) and (r["alpha_p"] == -100).all()
    assert (r["neighbor_q"] == 0).all() and (r["label_q"] == -100).all()
    # stars scaled to 1e-3: every area falls under the absolute tolerance, so the P-side and
    # Q-side counts differ and the pair is invalid (no arrays)
    P, Q = synth.random_star_pairs(7, 1, 4, 12, spread=1.0)[0]
    r = pyoracle.pair_intersections(P * 1e-3, Q * 1e-3)
    assert r["invalid"] == 1 and r["status"] == 1
    assert "xy_p" not in r and r["n_p"] >= len(P) and r["n_q"] >= len(Q)


@pytest.mark.parametrize("name", ["Fig18", "Fig19"])
@pytest.mark.parametrize("gpu_semantics", [False, True])
def test_multi_component_figs_byte_identical(name, gpu_semantics):
    """Fig18 (6 x 10 rings, holes) and Fig19 (5 rings): every component of both inputs,
    against the reference's own clipper run here."""
    P = load_poly(_fig(name, "P.poly"))
    Q = load_poly(_fig(name, "Q.poly"))
    assert len(P) > 1
    r = pyoracle.clip_multi(P, Q, gpu_semantics=gpu_semantics)
    assert r.status[0] == 0
    assert format_reference(r.components(0)) == open(_fig(name, "R.run.poly")).read()


@pytest.mark.parametrize("union", [False, True])
def test_multi_component_matches_reference_clipper(union):
    from conftest import unpack_multi
    pairs, inter, uni = unpack_multi(os.path.join(GOLDEN, "holed_pairs.npz"))
    assert len(pairs) == 150 and sum(len(p) for p, _ in pairs) > 300
    for (P, Q), exp in zip(pairs, uni if union else inter):
        for gs in (False, True):
            r = pyoracle.clip_multi(P, Q, union=union, gpu_semantics=gs)
            assert r.status[0] == 0
            assert same_components(r.components(0), exp)


def test_multi_component_single_rings_equal_single_pair():
    """One ring per side: the multi-component clipper gives what the single-pair one does."""
    pairs, expect = unpack_pairs(os.path.join(GOLDEN, "random_pairs.npz"))
    for (P, Q), _ in list(zip(pairs, expect))[:150]:
        a = pyoracle.clip_pair(P, Q)
        b = pyoracle.clip_multi([P], [Q])
        assert a.status[0] == b.status[0]
        if a.status[0] == 0:
            assert same_components(a.components(0), b.components(0))
