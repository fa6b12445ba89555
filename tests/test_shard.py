"""Slab sharding across ranks (gcmfgh.shard) with world size 2 over gloo on the CPU: each
rank joins and clips its x-slab of base polygons against the whole overlay layer (the
oracle stands in for the per-rank GPU compute here), the results are gathered with one
all_gather of counts and one of padded arrays, and the merge equals the unsharded result
exactly.  Also covers a rank whose slab yields no pairs."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import pyoracle
from gcmfgh import shard, synth


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_join_clip(base, ovl):
    j = pyoracle.join(base, ovl)
    sel = j.clip == 1
    b, o = j.b[sel], j.o[sel]
    c = pyoracle.clip_batch(base, ovl, b, o)
    return b, o, c.ncomp, c.comp_size, c.xy


def _worker(rank, world, port, base, ovl, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sub, ids = shard.shard_base(base, world, rank)
        if sub.n_polys:
            b, o, nc, cs, xy = _oracle_join_clip(sub, ovl)
            b = ids[b]
        else:
            b = o = nc = cs = np.zeros(0, np.int32)
            xy = np.zeros(0)
        merged = shard.gather_results(dist, b, o, nc, cs, xy)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), *merged, n_local=len(b))
    finally:
        dist.destroy_process_group()


def _run(world, base, ovl, tmp_path):
    mp.spawn(_worker, args=(world, _free_port(), base, ovl, str(tmp_path)), nprocs=world, join=True)
    return [np.load(tmp_path / f"r{r}.npz") for r in range(world)]


def test_two_rank_slabs_equal_single_process(tmp_path):
    base, ovl = synth.small_join(0, 2000)
    want = _oracle_join_clip(base, ovl)
    outs = _run(2, base, ovl, tmp_path)
    for d in outs:                                   # every rank holds the merged result
        got = [d[f"arr_{i}"] for i in range(5)]
        for g, w in zip(got, want):
            assert np.array_equal(np.asarray(g), np.asarray(w))
    assert all(int(d["n_local"]) > 0 for d in outs)


def test_rank_with_an_empty_slab(tmp_path):
    """The base polygons of the upper x-slab are moved far from every overlay polygon: that
    rank finds no pairs and still takes part in the gather."""
    base, ovl = synth.small_join(0, 300)
    x1 = shard.layer_mbr_x1(base)
    far = x1 >= np.median(x1)
    rings = [base.ring(i) + (np.array([1e6, 0.0]) if far[i] else 0.0) for i in range(base.n_polys)]
    base2 = synth.Layer.from_rings(rings)
    want = _oracle_join_clip(base2, ovl)
    outs = _run(2, base2, ovl, tmp_path)
    assert int(outs[1]["n_local"]) == 0 and int(outs[0]["n_local"]) > 0
    for d in outs:
        got = [d[f"arr_{i}"] for i in range(5)]
        for g, w in zip(got, want):
            assert np.array_equal(np.asarray(g), np.asarray(w))


def test_slab_partition_is_a_partition():
    base, _ = synth.small_join(0, 2000)
    seen = np.zeros(base.n_polys, int)
    for r in range(3):
        _, ids = shard.shard_base(base, 3, r)
        seen[ids] += 1
    assert (seen == 1).all()


def test_merge_results_orders_pairs_and_their_vertices():
    """Two parts with interleaved (b, o) keys: the merge sorts pairs and carries each pair's
    components and vertices along, empty pairs included."""
    p0 = (np.array([5, 1]), np.array([0, 2]), np.array([2, 0]), np.array([3, 1]),
          np.arange(8, dtype=float))                            # pair (5,0): comps of 3 and 1 vertices
    p1 = (np.array([3]), np.array([7]), np.array([1]), np.array([2]), np.array([100., 101., 102., 103.]))
    b, o, nc, cs, xy = shard.merge_results([p0, p1])
    assert list(zip(b, o)) == [(1, 2), (3, 7), (5, 0)]
    assert list(nc) == [0, 1, 2] and list(cs) == [2, 3, 1]
    assert list(xy) == [100., 101., 102., 103.] + list(np.arange(8, dtype=float))


def test_subset_layer_matches_rings():
    base, _ = synth.small_join(0, 200)
    ids = np.array([7, 3, 150, 0])
    sub = shard.subset_layer(base, ids)
    for k, i in enumerate(ids):
        assert np.array_equal(sub.ring(k), base.ring(int(i)))
