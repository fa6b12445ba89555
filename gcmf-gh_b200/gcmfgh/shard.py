"""Slab sharding of the join-and-clip across ranks (one process per GPU).

The path has no exchange step inside it: the MBR candidate predicate, the filters and the
clip each look at one (base, overlay) pair.  So base polygons are split into x-slabs by
their MBR x1 (the key the sweep sorts on, GPU_MBR.h:339-539), each rank joins and clips
its slab against the whole overlay layer, and the only collective is the gather of the
per-rank results at the end: one all_gather of the three counts (pairs, components,
vertices), then one all_gather of the padded result arrays.  Sorting the gathered pairs
by (base, overlay) reproduces the single-process result exactly, because every pair is
computed by exactly one rank with the same arithmetic.

Everything here is host logic over numpy/torch; the per-rank compute is passed in, so the
same code runs over NCCL with the CUDA engine and over gloo with the oracle.
"""
from __future__ import annotations

import numpy as np

from . import synth


def layer_mbr_x1(layer: synth.Layer) -> np.ndarray:
    """x1 of every polygon's MBR over its stored vertices (closing vertex included)."""
    xs = layer.xy[0::2]
    starts = (layer.vps - layer.vnum).astype(np.int64)
    out = np.full(layer.n_polys, np.inf)
    nz = layer.vnum > 0
    out[nz] = np.minimum.reduceat(xs, starts[nz]) if nz.any() else out[nz]
    return out


def slab_edges(x1: np.ndarray, world: int) -> np.ndarray:
    """world+1 slab boundaries at x1 quantiles (equal polygon counts per slab)."""
    finite = np.sort(x1[np.isfinite(x1)])
    if finite.size == 0:
        return np.concatenate([[-np.inf], np.full(world - 1, np.inf), [np.inf]])
    qs = [finite[min(len(finite) - 1, (len(finite) * r) // world)] for r in range(1, world)]
    return np.concatenate([[-np.inf], qs, [np.inf]])


def ranges_to_index(starts: np.ndarray, lens: np.ndarray) -> np.ndarray:
    """Concatenation of the index ranges [starts[i], starts[i] + lens[i])."""
    starts = np.asarray(starts, np.int64)
    lens = np.asarray(lens, np.int64)
    total = int(lens.sum())
    if total == 0:
        return np.zeros(0, np.int64)
    first = np.cumsum(lens) - lens
    return np.arange(total, dtype=np.int64) - np.repeat(first, lens) + np.repeat(starts, lens)


def subset_layer(layer: synth.Layer, ids: np.ndarray) -> synth.Layer:
    """The listed polygons of a layer, in the given order, as a layer of their own."""
    ids = np.asarray(ids, np.int64)
    vn = layer.vnum[ids].astype(np.int64)
    v = ranges_to_index(layer.vps[ids] - vn, vn)
    xy = layer.xy.reshape(-1, 2)[v]
    return synth.Layer(xy, vn.astype(np.int32))


def shard_base(layer: synth.Layer, world: int, rank: int):
    """(sub-layer of this rank's base polygons, their global ids)."""
    x1 = layer_mbr_x1(layer)
    edges = slab_edges(x1, world)
    owner = np.searchsorted(edges, x1, side="right") - 1
    owner = np.clip(owner, 0, world - 1)
    ids = np.flatnonzero(owner == rank).astype(np.int32)
    return subset_layer(layer, ids), ids


def merge_results(parts):
    """Merges per-rank results [(b, o, ncomp, comp_size, xy), ...] (b global base ids) into
    one result sorted by (b, o): (b, o, ncomp, comp_size, xy).  Vectorised: one sort of
    the pairs, then the components and vertices of every pair gathered by index ranges."""
    B = np.concatenate([np.asarray(p[0], np.int64) for p in parts]) if parts else np.zeros(0, np.int64)
    O = np.concatenate([np.asarray(p[1], np.int64) for p in parts]) if parts else np.zeros(0, np.int64)
    N = np.concatenate([np.asarray(p[2], np.int64) for p in parts]) if parts else np.zeros(0, np.int64)
    S = np.concatenate([np.asarray(p[3], np.int64) for p in parts]) if parts else np.zeros(0, np.int64)
    X = np.concatenate([np.asarray(p[4], np.float64) for p in parts]) if parts else np.zeros(0)
    cstart = np.cumsum(N) - N                              # first component of each pair
    vcomp = np.cumsum(S) - S                               # first vertex of each component
    vpair = np.zeros(len(N), np.int64)                     # first vertex and vertex count per pair
    nz = N > 0
    vpair[nz] = vcomp[cstart[nz]]
    vlen = np.add.reduceat(S, cstart[nz]) if nz.any() else np.zeros(0, np.int64)
    vl = np.zeros(len(N), np.int64)
    vl[nz] = vlen
    order = np.lexsort((O, B))
    comps = ranges_to_index(cstart[order], N[order])
    verts = ranges_to_index(vpair[order], vl[order])
    xy = X.reshape(-1, 2)[verts].reshape(-1) if len(verts) else np.zeros(0)
    return (B[order].astype(np.int32), O[order].astype(np.int32), N[order].astype(np.int32),
            S[comps].astype(np.int32), xy)


def _all_gather_padded(dist, t, n_all, device):
    import torch
    cap = max(int(n_all.max()), 1)
    pad = torch.zeros(cap, dtype=t.dtype, device=device)
    pad[: t.numel()] = t
    outs = [torch.zeros(cap, dtype=t.dtype, device=device) for _ in range(len(n_all))]
    dist.all_gather(outs, pad)
    return [o[: int(n)].cpu().numpy() for o, n in zip(outs, n_all)]


def gather_results(dist, b, o, ncomp, comp_size, xy, device="cpu"):
    """All ranks call this with their pairs (global base id b, overlay id o, components per
    pair, component sizes, vertices).  Returns the merged result sorted by (b, o) on every
    rank: (b, o, ncomp, comp_size, xy)."""
    import torch
    counts = torch.tensor([len(b), len(comp_size), len(xy)], dtype=torch.int64, device=device)
    allc = [torch.zeros(3, dtype=torch.int64, device=device) for _ in range(dist.get_world_size())]
    dist.all_gather(allc, counts)
    allc = np.stack([c.cpu().numpy() for c in allc])
    tb = _all_gather_padded(dist, torch.as_tensor(np.asarray(b, np.int64), device=device), allc[:, 0], device)
    to = _all_gather_padded(dist, torch.as_tensor(np.asarray(o, np.int64), device=device), allc[:, 0], device)
    tn = _all_gather_padded(dist, torch.as_tensor(np.asarray(ncomp, np.int64), device=device), allc[:, 0], device)
    ts = _all_gather_padded(dist, torch.as_tensor(np.asarray(comp_size, np.int64), device=device), allc[:, 1],
                            device)
    tx = _all_gather_padded(dist, torch.as_tensor(np.asarray(xy, np.float64), device=device), allc[:, 2], device)
    return merge_results([(tb[r], to[r], tn[r], ts[r], tx[r]) for r in range(len(tb))])
