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


def shard_base(layer: synth.Layer, world: int, rank: int):
    """(sub-layer of this rank's base polygons, their global ids)."""
    x1 = layer_mbr_x1(layer)
    edges = slab_edges(x1, world)
    owner = np.searchsorted(edges, x1, side="right") - 1
    owner = np.clip(owner, 0, world - 1)
    ids = np.flatnonzero(owner == rank).astype(np.int32)
    sub = synth.Layer.from_rings([layer.ring(int(i)) for i in ids])
    return sub, ids


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
    # per pair: its components and vertices, then reorder by (b, o)
    rows = []
    for r in range(len(tb)):
        cbase = np.concatenate([[0], np.cumsum(tn[r])]).astype(np.int64)
        vstart = np.concatenate([[0], np.cumsum(2 * ts[r])]).astype(np.int64)
        for k in range(len(tb[r])):
            c0, c1 = cbase[k], cbase[k + 1]
            rows.append((int(tb[r][k]), int(to[r][k]), ts[r][c0:c1], tx[r][vstart[c0]:vstart[c1]]))
    rows.sort(key=lambda t: (t[0], t[1]))
    mb = np.array([t[0] for t in rows], np.int32)
    mo = np.array([t[1] for t in rows], np.int32)
    mn = np.array([len(t[2]) for t in rows], np.int32)
    ms = np.concatenate([t[2] for t in rows]).astype(np.int32) if rows else np.zeros(0, np.int32)
    mx = np.concatenate([t[3] for t in rows]) if rows else np.zeros(0)
    return mb, mo, mn, ms, mx
