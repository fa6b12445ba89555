"""GPU parity of the GCMF join (MBR filter, common MBR, containment, common-MBR edge
filter, segment refine, clip set) and of the end-to-end join+clip against the oracle.
Candidate sets, flags and counts are integer results and must be identical."""
import numpy as np
import pytest

import pyoracle
from gcmfgh import synth

pytestmark = pytest.mark.gpu

FIELDS = ["b", "o", "cmbr", "pip_type", "pip_flag", "join_flag", "bE", "oE", "seg_flag", "clip"]


def _join_equal(engine, base, ovl):
    import gcmfgh
    db, do = gcmfgh.DeviceLayer(base), gcmfgh.DeviceLayer(ovl)
    info = engine.join(db, do)
    o = pyoracle.join(base, ovl)
    for f in FIELDS:
        assert np.array_equal(engine.join_field(f).reshape(-1), np.asarray(getattr(o, f)).reshape(-1)), f
    assert np.array_equal(engine.join_field("valid_b"), o.valid_b)
    assert np.array_equal(engine.join_field("mbr_b"), o.mbr_b)
    assert info["n_pairs"] == len(o.b)
    assert info["n_clip"] == int(o.clip.sum())
    assert info["n_within"] == int(o.pip_flag.sum()) and info["n_seg"] == int(o.seg_flag.sum())
    return db, do, info, o


def _clip_equal(engine, db, do, base, ovl):
    info = engine.clip_joined(db, do)
    r = engine.clip_result()
    cb, co = engine.join_field("clip_b"), engine.join_field("clip_o")
    o = pyoracle.clip_batch(base, ovl, cb, co)
    assert engine.last_device_error() == 0
    assert np.array_equal(r.status, o.status)
    assert np.array_equal(r.count1, o.count1)
    assert np.array_equal(r.ncomp, o.ncomp)
    assert np.array_equal(r.comp_size, o.comp_size)
    assert np.array_equal(r.xy, o.xy)
    return info, r


def test_small_join_and_clip(engine):
    base, ovl = synth.small_join()
    db, do, info, _ = _join_equal(engine, base, ovl)
    assert info["n_pairs"] == 1813
    _clip_equal(engine, db, do, base, ovl)


def test_batched_join_and_clip_full_size(engine):
    """The full 200,000 x 200,000 polygon workload: every candidate, flag and clipped
    vertex against the oracle."""
    base, ovl = synth.batched_join()
    db, do, info, _ = _join_equal(engine, base, ovl)
    assert info["n_pairs"] > 500000 and info["n_clip"] > 400000
    cinfo, r = _clip_equal(engine, db, do, base, ovl)
    assert cinfo["n_error"] == 0


def _box(x1, y1, x2, y2):
    return np.array([[x1, y1], [x2, y1], [x2, y2], [x1, y2]], dtype=np.float64)


def test_touching_mbrs_tie_rule(engine):
    base = synth.Layer.from_rings([_box(0, 0, 1, 1), np.array([[0, 0], [0, 1], [0, 2]], float)])
    ovl = synth.Layer.from_rings([_box(1, 0, 2, 1), _box(-1, 0, 0, 1), _box(0, 1, 1, 2),
                                  _box(0.5, 0.5, 3, 3), _box(1, 1, 2, 2), _box(5, 5, 6, 6)])
    _, _, info, o = _join_equal(engine, base, ovl)
    assert list(zip(o.b, o.o)) == [(0, 1), (0, 2), (0, 3)]


def test_containment_and_duplicates(engine):
    rings = [_box(0, 0, 10, 10), _box(20, 20, 30, 30), _box(2, 2, 3, 3), _box(2, 2, 3, 3)]
    base = synth.Layer.from_rings(rings)
    ovl = synth.Layer.from_rings(rings[::-1] + [_box(25, 15, 35, 25)])
    db, do, info, o = _join_equal(engine, base, ovl)
    assert info["n_within"] > 0
    _clip_equal(engine, db, do, base, ovl)


def test_single_and_empty_layers(engine):
    import gcmfgh
    one = synth.Layer.from_rings([_box(0, 0, 1, 1)])
    _join_equal(engine, one, one)
    empty = synth.Layer(np.zeros((0, 2)), np.zeros(0, np.int32))
    db, do = gcmfgh.DeviceLayer(one), gcmfgh.DeviceLayer(empty)
    info = engine.join(db, do)
    assert info["n_pairs"] == 0 and info["n_clip"] == 0


@pytest.mark.parametrize("seed", [11, 12])
def test_dense_random_layers(engine, seed):
    """Many overlaps per polygon, varied sizes."""
    rng = np.random.default_rng(seed)
    layers = []
    for _ in range(2):
        n = 3000
        counts = rng.integers(3, 200, size=n)
        centres = rng.uniform(0, 300, size=(n, 2))
        radius = rng.lognormal(np.log(8.0), 0.6, size=n)
        layers.append(synth.star_layer(rng, counts, centres, radius))
    db, do, info, _ = _join_equal(engine, *layers)
    _clip_equal(engine, db, do, *layers)


def test_host_entry_point_equals_device_path(engine):
    base, ovl = synth.small_join(seed=3, n=1500)
    import gcmfgh
    db, do = gcmfgh.DeviceLayer(base), gcmfgh.DeviceLayer(ovl)
    ji = engine.join(db, do)
    ci = engine.clip_joined(db, do)
    xy = engine.clip_field("xy")
    ji2, ci2 = engine.join_clip_host(base, ovl)
    assert ji == ji2 and ci == ci2
    assert np.array_equal(engine.clip_field("xy"), xy)


@pytest.mark.parametrize("name", ["small_join", "dense"])
def test_join_matches_reference_gpu_join(engine, name, tmp_path):
    """The engine's join on the layers of tests/golden/join_ref_<name>.npz (read through
    the engine's text reader) against the reference's own GPU join stages run on the
    same text: candidates, common MBRs, containment, edge-filter counts, refine flags."""
    import os
    import gcmfgh
    from conftest import GOLDEN
    from golden import make_join_goldens as mjg
    fx = np.load(os.path.join(GOLDEN, f"join_ref_{name}.npz"))
    if "gpu_jxy" not in fx.files:
        pytest.skip("fixture made without the reference's GPU stages")
    pb, po = mjg.write_case_text(name, str(tmp_path))
    assert mjg.sha256(pb) == str(fx["text_sha_b"]) and mjg.sha256(po) == str(fx["text_sha_o"])
    base, _ = gcmfgh.read_text_layer(pb)
    ovl, _ = gcmfgh.read_text_layer(po)
    engine.join(gcmfgh.DeviceLayer(base), gcmfgh.DeviceLayer(ovl))
    r = mjg.reference_join_by_pair(fx)
    for f in ("b", "o", "pip_type", "pip_flag", "join_flag", "bE", "oE", "seg_flag"):
        assert np.array_equal(engine.join_field(f).astype(np.int64), r[f].astype(np.int64)), f
    assert np.array_equal(engine.join_field("cmbr").reshape(-1, 4), r["cmbr"])


def _near_tie_layers(seed=3, n=400):
    """Squares whose MBRs meet in y within a few FP64 ulps (far below one FP32 ulp): base
    i spans y in [0, 1 + d_i], overlay i spans [1 + e_i, 2], with d_i, e_i of order 1e-9,
    so the y overlap -- and the edges touching the common MBR -- are decided below FP32
    resolution; plus shifted copies and a few random stars around them."""
    rng = np.random.default_rng(seed)
    rb, ro = [], []
    for i in range(n):
        x = 3.0 * i
        d, e = rng.integers(-3, 4, size=2) * 1e-9
        top = 1.0 + d
        rb.append(np.array([[x, 0.0], [x + 1.0, 0.0], [x + 1.0, top], [x, top]]))
        ro.append(np.array([[x + 0.5, 1.0 + e], [x + 1.5, 1.0 + e], [x + 1.5, 2.0], [x + 0.5, 2.0]]))
        if i % 4 == 0:                                  # an edge ending a few ulps inside the CMBR
            u = np.nextafter(1.0 + e, 2.0) if i % 8 == 0 else np.nextafter(1.0 + e, 0.0)
            ro.append(np.array([[x + 0.2, u], [x + 0.8, 1.5], [x + 0.2, 1.9]]))
    stars_b, stars_o = synth.small_join(seed, 200)
    rb += [stars_b.ring(i) for i in range(stars_b.n_polys)]
    ro += [stars_o.ring(i) for i in range(stars_o.n_polys)]
    return synth.Layer.from_rings(rb), synth.Layer.from_rings(ro)


def test_fp32_prefilters_keep_fp64_results(engine):
    """The join's FP32 outward-rounded MBR and edge prefilters (GCMFGH_TUNE_F32_FILTER)
    give the FP64 tests' candidates, flags and edge counts on near-tie boxes."""
    base, ovl = _near_tie_layers()
    o = pyoracle.join(base, ovl)
    got = {}
    for f32 in (0, 1, 2, 3):
        engine.set_tuning(f32_filter=f32)
        try:
            _join_equal(engine, base, ovl)
            got[f32] = [engine.join_field(f).copy() for f in FIELDS]
        finally:
            engine.set_tuning(f32_filter=1)
    for f32 in (1, 2, 3):
        for a, b in zip(got[0], got[f32]):
            assert np.array_equal(a, b)
    assert int(o.pip_type.size) > 250          # about half the near-tie squares join


def _keys(engine, db, do):
    engine.join(db, do)
    return np.stack([engine.join_field("b").reshape(-1), engine.join_field("o").reshape(-1)])


@pytest.mark.parametrize("case", ["small", "ties", "huge_boxes", "listing_limit", "degenerate_extent"])
def test_grid_probe_equals_sort_sweep(engine, case):
    """The MBR filter's grid probe (default) and the reference's sort-sweep form the same
    candidate list: on a seeded layer pair; on boxes that touch at cell-size multiples; on
    layers where most boxes span the whole extent (a coarse grid, every cell listing
    them); on tiny boxes plus 500 boxes spanning everything (the listing passes its limit
    and the sweep takes over); and on a thin extent (all boxes in one row of cells)."""
    import gcmfgh
    rng = np.random.default_rng(5)
    if case == "small":
        base, ovl = synth.small_join(11, 3000)
    elif case == "ties":
        rings = [_box(x, y, x + 1, y + 1) for x in range(0, 40, 1) for y in range(0, 40, 2)]
        base = synth.Layer.from_rings(rings)
        ovl = synth.Layer.from_rings([_box(x + 1, y, x + 2, y + 1) for x in range(0, 40, 2) for y in range(0, 40)])
    elif case == "huge_boxes":
        small = [_box(*c, *(c + 1.0)) for c in rng.uniform(0, 100, size=(3000, 2))]
        huge = [_box(-1.0 - i, -1.0 - i, 101.0 + i, 101.0 + i) for i in range(2000)]
        base = synth.Layer.from_rings(small + huge[:5])
        ovl = synth.Layer.from_rings(huge + small[::3])
    elif case == "listing_limit":
        tiny = [_box(*c, *(c + 0.01)) for c in rng.uniform(0, 1000, size=(100000, 2))]
        huge = [_box(-1.0 - i, -1.0 - i, 1001.0 + i, 1001.0 + i) for i in range(500)]
        base = synth.Layer.from_rings(tiny[:3000] + huge[:3])
        ovl = synth.Layer.from_rings(tiny + huge)
    else:
        base = synth.Layer.from_rings([_box(x, 0, x + 1.5, 1e-9) for x in rng.uniform(0, 1000, 2000)])
        ovl = synth.Layer.from_rings([_box(x, 0, x + 0.5, 2e-9) for x in rng.uniform(0, 1000, 2000)])
    db, do = gcmfgh.DeviceLayer(base), gcmfgh.DeviceLayer(ovl)
    try:
        engine.set_tuning(join_sweep=False)
        grid = _keys(engine, db, do)
        engine.set_tuning(join_sweep=True)
        sweep = _keys(engine, db, do)
    finally:
        engine.set_tuning(join_sweep=True)             # the default
    assert grid.shape[1] > 0
    assert np.array_equal(grid, sweep)
    o = pyoracle.join(base, ovl)
    assert np.array_equal(grid[0], o.b) and np.array_equal(grid[1], o.o)


@pytest.mark.parametrize("run", [40, 200, 1000])
def test_sweep_sort_keys_equal_in_fp32(engine, run):
    """The sweep sorts 32-bit keys (x1 rounded down to FP32) and mends runs of equal keys to
    the exact (x1, id) order; runs longer than 256 send the layer to a 64-bit sort. Boxes
    whose x1 differ by 1e-9 near 1e5 share their FP32 key: runs of 40, 200 and 1,000, with
    and without equal x1, against the oracle's candidate list."""
    import gcmfgh
    rng = np.random.default_rng(run)
    x1 = 1e5 + rng.permutation(run) * 1e-9
    x1[: run // 4] = x1[0]                                # some equal x1 too
    base = synth.Layer.from_rings([_box(x, 0.0, x + 0.5, 1.0) for x in x1] +
                                  [_box(x, 0.0, x + 1.0, 1.0) for x in rng.uniform(0, 2e5, 300)])
    ovl = synth.Layer.from_rings([_box(x + 0.25, 0.5, x + 2.0, 2.0) for x in x1[::-1]] +
                                 [_box(x, 0.5, x + 1.0, 1.5) for x in rng.uniform(0, 2e5, 300)])
    engine.set_tuning(join_sweep=True)
    db, do = gcmfgh.DeviceLayer(base), gcmfgh.DeviceLayer(ovl)
    engine.join(db, do)
    o = pyoracle.join(base, ovl)
    assert len(o.b) > run
    assert np.array_equal(engine.join_field("b").reshape(-1), o.b)
    assert np.array_equal(engine.join_field("o").reshape(-1), o.o)


def test_clip_of_join_takes_join_edge_lists(engine):
    """gh_clip_joined takes each clip pair's common-MBR edge lists from the join (dropping
    the join's zero-length closing edge) when both rings are closed, and tests the edges
    itself otherwise: a layer pair with every tenth stored closing vertex moved off the
    first vertex gives the oracle's join and clip either way."""
    import gcmfgh
    base, ovl = synth.small_join(21, 3000)
    xy = base.xy.reshape(-1, 2).copy()
    for i in range(0, base.n_polys, 10):
        xy[int(base.vps[i]) - 1] += 1e-3                  # the stored closing vertex
    base = synth.Layer(xy, base.vnum)
    db, do, info, _ = _join_equal(engine, base, ovl)
    assert info["n_clip"] > 1000
    _clip_equal(engine, db, do, base, ovl)


def test_one_pass_sweep_and_filter_equal_two_pass_and_overflow(engine):
    """The join's one-pass sweep and common-MBR edge filter (default) against their
    count-then-write forms, on a small join and then on a larger one whose candidates and
    edge lists outnumber the arrays sized from the small join's totals (each pass runs
    again at the counted sizes); every join field and the clip against the oracle."""
    import gcmfgh
    for n in (2000, 40000):
        base, ovl = synth.small_join(31, n)
        db, do = gcmfgh.DeviceLayer(base), gcmfgh.DeviceLayer(ovl)
        info = engine.join(db, do)
        one = {f: engine.join_field(f).reshape(-1).copy() for f in FIELDS}
        engine.set_tuning(sweep_two_pass=True)
        try:
            info2 = engine.join(db, do)
            two = {f: engine.join_field(f).reshape(-1).copy() for f in FIELDS}
        finally:
            engine.set_tuning(sweep_two_pass=False)
        assert info == info2
        for f in FIELDS:
            assert np.array_equal(one[f], two[f]), f
        db, do, info, _ = _join_equal(engine, base, ovl)
        if n == 2000:
            _clip_equal(engine, db, do, base, ovl)
    assert info["n_pairs"] > 2000 * 1.25 + 65536
