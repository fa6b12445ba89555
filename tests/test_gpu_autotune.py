"""The work-distribution autotuner (gcmfgh_autotune_joined): it records the fastest
thresholds for the workload's signature, later clips of the same signature use them, the
results are bit-identical to those under the default thresholds, and the records survive
a new context through the file named by GCMFGH_TUNING_FILE."""
import os

import numpy as np
import pytest

from gcmfgh import synth

pytestmark = pytest.mark.gpu


def _clip(eng, db, do):
    eng.join(db, do)
    eng.clip_joined(db, do)
    r = eng.clip_result()
    return r.status, r.ncomp, r.comp_size, r.xy


def test_autotune_records_and_keeps_results(tmp_path, monkeypatch):
    import gcmfgh
    path = tmp_path / "tuning.jsonl"
    monkeypatch.setenv("GCMFGH_TUNING_FILE", str(path))
    base, ovl = synth.batched_join(seed=2, n=20_000)
    eng = gcmfgh.Engine(0)
    try:
        db, do = gcmfgh.DeviceLayer(base), gcmfgh.DeviceLayer(ovl)
        want = _clip(eng, db, do)
        n = eng.join(db, do)["n_clip"]
        before = eng.tuning_for(db, do, n)
        t = eng.autotune_joined(db, do)
        assert t["configs_timed"] >= 10
        assert t["ms_tuned"] <= t["ms_default"]
        assert t["pairs_log2"] == int(np.floor(np.log2(n)))
        now = eng.tuning_for(db, do, n)
        for k in ("bin_grid", "tile_label", "mid_label", "wide_label"):
            assert now[k] == t[k]
        assert before["bin_grid"] == 1 << 16                # defaults before tuning
        for g, w in zip(_clip(eng, db, do), want):          # same results under the tuned limits
            assert np.array_equal(g, w)
    finally:
        eng.close()
    assert path.exists() and "bin_grid" in path.read_text()
    eng2 = gcmfgh.Engine(0)                                  # a new context reads the records
    try:
        db, do = gcmfgh.DeviceLayer(base), gcmfgh.DeviceLayer(ovl)
        again = eng2.tuning_for(db, do, n)
        for k in ("bin_grid", "tile_label", "mid_label", "wide_label", "ms_tuned"):
            assert again[k] == pytest.approx(t[k], abs=1e-3)
        eng2.set_tuning(bin_grid=12345)                     # explicit settings win
        assert eng2.tuning_for(db, do, n)["bin_grid"] == 12345
    finally:
        eng2.close()
