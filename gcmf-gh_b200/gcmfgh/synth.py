"""Seeded synthetic polygon layers for the join-and-clip workloads.

Layers are returned in the reference's join layout (spatialJoin3.cu:205-212,
SEQ_Overlay.h:352-380): interleaved FP64 coordinates with each polygon's closing
vertex stored, ``vnum`` = vertex count including the closing vertex, ``vps`` = its
inclusive prefix sum.  Star polygons (vertices at sorted uniform angles around a
centre, counter-clockwise) are simple by construction.

Workloads (all FP64):
  * ``small_join``: two layers of 2,000 stars, seed 0; vertex count U{8..64};
    centre U[0,1000]^2; base radius log-normal(ln 5, 0.5); radius = base*U(0.6,1.0).
  * ``large_pair``: one 1,000,000-vertex star (radius U(0.8,1.2), centre 0,0) and one
    500,000-vertex star (radius U(0.7,1.3), centre (0.05,0.03)), seed 1.
  * ``batched_join``: two layers of 200,000 stars, seed 2; vertex count
    floor(Pareto(alpha=1.5, x_m=4)) capped at 100,000; centres from a 64-component
    Gaussian mixture over [0,1e5]^2 (sigma 2,000, means U[0,1e5]^2); base radius
    log-normal(ln 50, 0.7); radius = base*U(0.6,1.0).
"""
from __future__ import annotations

import numpy as np


class Layer:
    """One polygon layer in the reference layout (closing vertex stored)."""

    def __init__(self, xy: np.ndarray, vnum: np.ndarray):
        self.xy = np.ascontiguousarray(xy, dtype=np.float64).reshape(-1)
        self.vnum = np.ascontiguousarray(vnum, dtype=np.int32)
        self.vps = np.cumsum(self.vnum, dtype=np.int64)

    @property
    def n_polys(self) -> int:
        return int(self.vnum.shape[0])

    @property
    def n_vertices(self) -> int:
        return int(self.vps[-1]) if self.vnum.shape[0] else 0

    def ring(self, i: int) -> np.ndarray:
        """Open ring (n x 2) of polygon i, closing vertex dropped."""
        end = int(self.vps[i])
        start = end - int(self.vnum[i])
        return self.xy[2 * start:2 * (end - 1)].reshape(-1, 2)

    @staticmethod
    def from_rings(rings) -> "Layer":
        vnum = np.array([len(r) + 1 for r in rings], dtype=np.int32)
        parts = []
        for r in rings:
            r = np.asarray(r, dtype=np.float64).reshape(-1, 2)
            parts.append(np.vstack([r, r[:1]]))
        xy = np.vstack(parts) if parts else np.zeros((0, 2))
        return Layer(xy, vnum)


def star_layer(rng: np.random.Generator, counts: np.ndarray, centres: np.ndarray,
               base_r: np.ndarray, rmin: float = 0.6, rmax: float = 1.0) -> Layer:
    """Vectorised star polygons: per polygon, sorted U[0,2pi) angles and radius
    base*U(rmin,rmax); the closing vertex repeats the first."""
    counts = np.asarray(counts, dtype=np.int64)
    n = counts.shape[0]
    total = int(counts.sum())
    pid = np.repeat(np.arange(n), counts)
    ang = rng.uniform(0.0, 2.0 * np.pi, size=total)
    # sort angles within each polygon: key = polygon id + angle/(2pi)
    order = np.lexsort((ang, pid))
    ang = ang[order]
    rad = np.repeat(base_r, counts) * rng.uniform(rmin, rmax, size=total)
    x = np.repeat(centres[:, 0], counts) + rad * np.cos(ang)
    y = np.repeat(centres[:, 1], counts) + rad * np.sin(ang)
    # insert the closing vertex after each polygon
    vnum = counts + 1
    ends = np.cumsum(vnum)
    starts = ends - vnum
    out = np.empty((int(ends[-1]) if n else 0, 2), dtype=np.float64)
    mask = np.ones(out.shape[0], dtype=bool)
    mask[ends - 1] = False
    out[mask, 0] = x
    out[mask, 1] = y
    out[ends - 1] = out[starts]
    return Layer(out, vnum.astype(np.int32))


def small_join(seed: int = 0, n: int = 2000):
    rng = np.random.default_rng(seed)
    layers = []
    for _ in range(2):
        counts = rng.integers(8, 65, size=n)
        centres = rng.uniform(0.0, 1000.0, size=(n, 2))
        base = rng.lognormal(np.log(5.0), 0.5, size=n)
        layers.append(star_layer(rng, counts, centres, base))
    return layers[0], layers[1]


def large_pair(seed: int = 1, n_subject: int = 1_000_000, n_clip: int = 500_000):
    rng = np.random.default_rng(seed)
    subj = star_layer(rng, np.array([n_subject]), np.array([[0.0, 0.0]]), np.array([1.0]), 0.8, 1.2)
    clip = star_layer(rng, np.array([n_clip]), np.array([[0.05, 0.03]]), np.array([1.0]), 0.7, 1.3)
    return subj, clip


def batched_join(seed: int = 2, n: int = 200_000, components: int = 64,
                 extent: float = 1e5, sigma: float = 2000.0, cap: int = 100_000):
    rng = np.random.default_rng(seed)
    means = rng.uniform(0.0, extent, size=(components, 2))
    layers = []
    for _ in range(2):
        counts = np.minimum(np.floor(4.0 * (1.0 + rng.pareto(1.5, size=n))), cap).astype(np.int64)
        comp = rng.integers(0, components, size=n)
        centres = means[comp] + rng.normal(0.0, sigma, size=(n, 2))
        base = rng.lognormal(np.log(50.0), 0.7, size=n)
        layers.append(star_layer(rng, counts, centres, base))
    return layers[0], layers[1]


def random_star_pairs(seed: int, npairs: int, vmin: int = 3, vmax: int = 40,
                      spread: float = 1.0):
    """Independent star pairs near the origin, for clip parity tests."""
    rng = np.random.default_rng(seed)
    pairs = []
    for _ in range(npairs):
        nv = rng.integers(vmin, vmax + 1, size=2)
        ps = []
        for k in range(2):
            ang = np.sort(rng.uniform(0.0, 2 * np.pi, size=nv[k]))
            r = rng.uniform(0.3, 1.0, size=nv[k])
            c = rng.uniform(-0.5 * spread, 0.5 * spread, size=2)
            ps.append(np.stack([c[0] + r * np.cos(ang), c[1] + r * np.sin(ang)], axis=1))
        pairs.append((ps[0], ps[1]))
    return pairs


def _star(rng, n, cx, cy, R, rlo=0.6, rhi=1.0):
    ang = np.sort(rng.uniform(0.0, 2 * np.pi, size=n))
    r = R * rng.uniform(rlo, rhi, size=n)
    return np.stack([cx + r * np.cos(ang), cy + r * np.sin(ang)], axis=1)


def degeneracy_pairs(seed: int = 3, npairs: int = 1_000_000, vmin: int = 4, vmax: int = 10_000,
                     quantum: float = 2.0 ** -20):
    """Independent pairs for the precision path, as (classes, [(P, Q), ...]).

    Vertex counts are log-uniform on [vmin, vmax] per polygon; centres uniform on
    [0, 1000]^2, radius 10 * U(0.6, 1.0) per vertex, counter-clockwise.  Classes (drawn
    per pair): 1 (2%) the overlay shares one vertex exactly with the base; 2 (1%) the
    overlay is the base translated along one of its edges by a quarter of that edge, so
    the two copies of the edge are collinear and overlap; 3 (1%) the overlay is the base
    translated by 1e-12 relative to its coordinates; 0 the rest, generic overlaps.  Classes
    1 and 2 use coordinates that are multiples of `quantum`, which makes both
    constructions exact in FP64."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(vmin), np.log(vmax + 1)
    classes = np.zeros(npairs, np.int8)
    pairs = []
    for k in range(npairs):
        nP, nQ = (int(v) for v in np.exp(rng.uniform(lo, hi, size=2)))
        nP, nQ = min(max(nP, vmin), vmax), min(max(nQ, vmin), vmax)
        u = rng.uniform()
        c = rng.uniform(0.0, 1000.0, size=2)
        P = _star(rng, nP, c[0], c[1], 10.0)
        if u < 0.02:
            classes[k] = 1
            P = np.round(P / quantum) * quantum
            Q = _star(rng, nQ, c[0] + rng.uniform(-8, 8), c[1] + rng.uniform(-8, 8), 10.0)
            Q = np.round(Q / quantum) * quantum
            i, j = int(rng.integers(nP)), int(rng.integers(nQ))
            Q = Q + (P[i] - Q[j])
        elif u < 0.03:
            classes[k] = 2
            P = np.round(P / quantum) * quantum
            i = int(rng.integers(nP))
            Q = P + 0.25 * (P[(i + 1) % nP] - P[i])
        elif u < 0.04:
            classes[k] = 3
            Q = P + 1e-12 * np.abs(P).max()
        else:
            Q = _star(rng, nQ, c[0] + rng.uniform(-10, 10), c[1] + rng.uniform(-10, 10), 10.0)
        pairs.append((P, Q))
    return classes, pairs


def serving_workload(seed: int = 4, n: int = 1_000_000, n_queries: int = 512, components: int = 64,
                     extent: float = 1e5, sigma: float = 2000.0, cap: int = 100_000,
                     qmin: int = 16, qmax: int = 50_000):
    """Resident layer of n stars with the batched workload's distributions (Pareto(1.5, 4)
    vertex counts capped at `cap`, 64-component GMM centres, log-normal(ln 50, 0.7) radius),
    and a pool of query stars whose vertex counts are log-uniform on [qmin, qmax], centred
    by the same mixture with the same radius law.  Returns (resident Layer, [query rings])."""
    rng = np.random.default_rng(seed)
    means = rng.uniform(0.0, extent, size=(components, 2))
    counts = np.minimum(np.floor(4.0 * (1.0 + rng.pareto(1.5, size=n))), cap).astype(np.int64)
    comp = rng.integers(0, components, size=n)
    centres = means[comp] + rng.normal(0.0, sigma, size=(n, 2))
    base = rng.lognormal(np.log(50.0), 0.7, size=n)
    resident = star_layer(rng, counts, centres, base)
    qcounts = np.exp(rng.uniform(np.log(qmin), np.log(qmax + 1), size=n_queries)).astype(np.int64)
    qcounts = np.clip(qcounts, qmin, qmax)
    qcomp = rng.integers(0, components, size=n_queries)
    qcentres = means[qcomp] + rng.normal(0.0, sigma, size=(n_queries, 2))
    qbase = rng.lognormal(np.log(50.0), 0.7, size=n_queries)
    ql = star_layer(rng, qcounts, qcentres, qbase)
    queries = [np.ascontiguousarray(ql.ring(i)) for i in range(n_queries)]
    return resident, queries


def holed_polygon(rng, cx, cy, vmin=5, vmax=30, max_holes=3, max_islands=2):
    """A multi-component polygon as a list of open rings: 1..max_islands disjoint star
    islands (radius 1), each with 0..max_holes star holes placed on a circle of radius 0.35
    around the island centre (hole radius <= 0.15, so holes are disjoint and inside).
    Holes are clockwise half of the time."""
    rings = []
    islands = int(rng.integers(1, max_islands + 1))
    for k in range(islands):
        ox = cx + 2.2 * k
        rings.append(_star(rng, int(rng.integers(vmin, vmax + 1)), ox, cy, 1.0, 0.6, 1.0))
        h = int(rng.integers(0, max_holes + 1))
        for t in range(h):
            ang = 2 * np.pi * t / max(h, 1) + rng.uniform(-0.3, 0.3)
            hole = _star(rng, int(rng.integers(max(3, vmin // 2), max(4, vmax // 2) + 1)),
                         ox + 0.35 * np.cos(ang), cy + 0.35 * np.sin(ang), 0.15, 0.5, 1.0)
            rings.append(hole[::-1].copy() if rng.random() < 0.5 else hole)
    return rings


def holed_pairs(seed: int, npairs: int, vmin: int = 5, vmax: int = 30):
    """Seeded pairs of multi-component polygons (islands with holes) whose centres are at
    most 0.8 apart, for the multi-component clip."""
    rng = np.random.default_rng(seed)
    pairs = []
    for _ in range(npairs):
        P = holed_polygon(rng, 0.0, 0.0, vmin, vmax)
        d = rng.uniform(0.0, 0.8, size=2)
        Q = holed_polygon(rng, d[0], d[1], vmin, vmax)
        pairs.append((P, Q))
    return pairs


def degeneracy_chunk_device(seed: int, chunk: int, npairs: int, device="cuda:0", vmin: int = 4,
                            vmax: int = 10_000, quantum: float = 2.0 ** -20):
    """One chunk of the degeneracy-stressed batch, generated on the GPU with torch (the
    million-pair batch does not fit the host loop of degeneracy_pairs): the same
    distributions and classes as degeneracy_pairs, from the seeded stream (seed, chunk).

    Vertex counts log-uniform on [vmin, vmax]; centres uniform on [0, 1000]^2; radius
    10 * U(0.6, 1.0) per vertex at sorted uniform angles (counter-clockwise); class 1 (2%):
    both polygons on the `quantum` lattice and the overlay translated so that one of its
    vertices equals one of the base's; class 2 (1%): the base on the lattice and the
    overlay = base translated along one of its edges by a quarter of that edge (collinear
    overlapping edges, same vertex count); class 3 (1%): overlay = base translated by
    1e-12 x max |coordinate|; class 0: an independent star centred within +-10.
    Returns (classes int8 numpy, base (xy, vnum, vps), overlay (xy, vnum, vps)) with the
    layers as device tensors in the layer layout (closing vertex stored)."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(int(seed) * 1_000_003 + int(chunk))
    f64 = dict(dtype=torch.float64, device=device)
    lo, hi = np.log(vmin), np.log(vmax + 1)

    def U(*shape):
        return torch.rand(*shape, generator=g, **f64)

    n = npairs
    cnt = torch.exp(lo + (hi - lo) * U(n, 2)).floor().clamp_(vmin, vmax).to(torch.int64)
    u = U(n)
    cls = torch.zeros(n, dtype=torch.int8, device=device)
    cls[u < 0.04] = 3
    cls[u < 0.03] = 2
    cls[u < 0.02] = 1
    cnt[:, 1] = torch.where((cls == 2) | (cls == 3), cnt[:, 0], cnt[:, 1])
    centre = 1000.0 * U(n, 2)
    off = torch.where((cls == 1).unsqueeze(1), 16.0 * U(n, 2) - 8.0, 20.0 * U(n, 2) - 10.0)

    def stars(counts, centres):
        tot = int(counts.sum())
        pid = torch.repeat_interleave(torch.arange(counts.numel(), device=device), counts)
        ang = 2.0 * np.pi * U(tot)
        order = torch.argsort(pid.to(torch.float64) + ang / (2.0 * np.pi + 1e-9))
        ang = ang[order]
        rad = 10.0 * (0.6 + 0.4 * U(tot))
        x = centres[pid, 0] + rad * torch.cos(ang)
        y = centres[pid, 1] + rad * torch.sin(ang)
        return torch.stack([x, y], 1), pid

    P, pidP = stars(cnt[:, 0], centre)
    Q, pidQ = stars(cnt[:, 1], centre + off)
    startP = torch.cumsum(cnt[:, 0], 0) - cnt[:, 0]
    startQ = torch.cumsum(cnt[:, 1], 0) - cnt[:, 1]
    lat = ((cls == 1) | (cls == 2))
    P = torch.where(lat[pidP].unsqueeze(1), torch.round(P / quantum) * quantum, P)
    Q = torch.where((cls == 1)[pidQ].unsqueeze(1), torch.round(Q / quantum) * quantum, Q)
    # class 1: translate Q so that Q[j] == P[i]
    i1 = (U(n) * cnt[:, 0]).floor().to(torch.int64).clamp_(max=cnt[:, 0] - 1)
    j1 = (U(n) * cnt[:, 1]).floor().to(torch.int64).clamp_(max=cnt[:, 1] - 1)
    shift1 = P[startP + i1] - Q[startQ + j1]
    # class 2: Q = P + 0.25 (P[i+1] - P[i]) (P's vertex count)
    i2 = (U(n) * cnt[:, 0]).floor().to(torch.int64).clamp_(max=cnt[:, 0] - 1)
    i2n = torch.where(i2 + 1 < cnt[:, 0], i2 + 1, torch.zeros_like(i2))
    shift2 = 0.25 * (P[startP + i2n] - P[startP + i2])
    # class 3: Q = P + 1e-12 max|P|
    amax = torch.zeros(n, **f64).scatter_reduce(0, pidP, P.abs().amax(1), reduce="amax", include_self=True)
    samePQ = ((cls == 2) | (cls == 3))[pidQ].unsqueeze(1)
    # for classes 2 and 3 the overlay's vertices are the base's, vertex for vertex
    local = torch.arange(Q.shape[0], device=device) - startQ[pidQ]
    Pfor = P[startP[pidQ] + torch.minimum(local, cnt[pidQ, 0] - 1)]
    Q = torch.where(samePQ, Pfor, Q)
    c = cls[pidQ].unsqueeze(1)
    Q = torch.where(c == 1, Q + shift1[pidQ], Q)
    Q = torch.where(c == 2, Q + shift2[pidQ], Q)
    Q = torch.where(c == 3, Q + (1e-12 * amax)[pidQ].unsqueeze(1), Q)

    def layer(V, counts, start):
        vnum = counts + 1
        ends = torch.cumsum(vnum, 0)
        xy = torch.empty(int(ends[-1]) if n else 0, 2, **f64)
        pos = torch.arange(V.shape[0], device=device)
        pid = torch.repeat_interleave(torch.arange(n, device=device), counts)
        xy[pos + pid] = V                                   # each polygon shifted by its closing vertices
        xy[ends - 1] = V[start]
        return xy.reshape(-1).contiguous(), vnum.to(torch.int32), ends.to(torch.int64)

    return cls.cpu().numpy(), layer(P, cnt[:, 0], startP), layer(Q, cnt[:, 1], startQ)
