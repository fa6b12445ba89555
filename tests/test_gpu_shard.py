"""Slab sharding driven by the CUDA engine.  The ranks of one workload run here one after
the other on the one GPU (their kernels never wait on each other, so nothing needs them
to run at the same time): each joins and clips its x-slab of base polygons against the
whole overlay layer, and the merge of the slabs' results equals the single-process
result bit for bit."""
import numpy as np
import pytest

from gcmfgh import shard, synth

pytestmark = pytest.mark.gpu


def _join_clip(engine, base, ovl):
    import gcmfgh
    db, do = gcmfgh.DeviceLayer(base), gcmfgh.DeviceLayer(ovl)
    engine.join(db, do)
    engine.clip_joined(db, do)
    r = engine.clip_result()
    return engine.join_field("clip_b"), engine.join_field("clip_o"), r.ncomp, r.comp_size, r.xy


@pytest.mark.parametrize("world", [2, 3])
def test_engine_slabs_merge_to_single_process_result(engine, world):
    base, ovl = synth.batched_join(seed=2, n=20_000)
    want = _join_clip(engine, base, ovl)
    parts = []
    for rank in range(world):
        sub, ids = shard.shard_base(base, world, rank)
        b, o, nc, cs, xy = _join_clip(engine, sub, ovl)
        parts.append((ids[b], o, nc, cs, xy))
        assert len(b) > 0
    got = shard.merge_results(parts)
    for g, w in zip(got, want):
        assert np.array_equal(np.asarray(g), np.asarray(w))
