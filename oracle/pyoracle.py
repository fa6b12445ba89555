"""ctypes front end of the CPU oracle (oracle/gcmfgh_oracle.cpp) and of the reference's
own sequential clipper binary (oracle/_ref/ghclip_ref).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg, as the checker.  The product library never imports it.
"""
from __future__ import annotations

import ctypes
import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libgcmfgh_oracle.so")
REF_BIN = os.path.join(HERE, "_ref", "ghclip_ref")

FLAG_UNION = 1
FLAG_GPU_SEMANTICS = 2
FLAG_EXACT = 4

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        d, i32, i64 = ctypes.c_double, ctypes.c_int, ctypes.c_int64
        vp = ctypes.c_void_p
        L.orc_clip_pair.argtypes = [vp, i32, vp, i32, d, d, i32]
        L.orc_clip_pair.restype = i32
        L.orc_clip_batch.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, i64, d, d, i32]
        L.orc_clip_batch.restype = i64
        L.orc_result_sizes.argtypes = [vp]
        L.orc_result_sizes.restype = i64
        L.orc_result_copy.argtypes = [vp] * 6
        L.orc_result_copy.restype = None
        L.orc_exact_signs.argtypes = [vp, i64, i32, vp]
        L.orc_exact_signs.restype = None
        L.orc_clip_multi.argtypes = [vp, vp, i32, vp, vp, i32, d, d, i32]
        L.orc_clip_multi.restype = i32
        L.orc_pair_intersections.argtypes = [vp, i32, vp, i32, d, i32, vp]
        L.orc_pair_intersections.restype = i32
        L.orc_pair_intersections_copy.argtypes = [vp] * 8
        L.orc_pair_intersections_copy.restype = None
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


class ClipResult:
    """Per-pair status, component lists and intersection counts."""

    def __init__(self, status, ncomp, count1, nrec, comp_size, xy):
        self.status = status
        self.ncomp = ncomp
        self.count1 = count1
        self.nrec = nrec
        self.comp_size = comp_size
        self.xy = xy
        self.comp_off = np.concatenate([[0], np.cumsum(comp_size, dtype=np.int64)])
        self.pair_comp_off = np.concatenate([[0], np.cumsum(ncomp, dtype=np.int64)])

    def components(self, k):
        out = []
        for c in range(self.pair_comp_off[k], self.pair_comp_off[k + 1]):
            a, b = self.comp_off[c], self.comp_off[c + 1]
            out.append(self.xy[2 * a:2 * b].reshape(-1, 2))
        return out


def _collect():
    L = lib()
    sz = np.zeros(3, dtype=np.int64)
    L.orc_result_sizes(_p(sz))
    npairs, ncomp, nv = (int(v) for v in sz)
    status = np.zeros(npairs, np.int32)
    ncmp = np.zeros(npairs, np.int32)
    count1 = np.zeros(npairs, np.int64)
    nrec = np.zeros(npairs, np.int64)
    csz = np.zeros(ncomp, np.int32)
    xy = np.zeros(2 * nv, np.float64)
    L.orc_result_copy(_p(status), _p(ncmp), _p(count1), _p(nrec), _p(csz), _p(xy))
    return ClipResult(status, ncmp, count1, nrec, csz, xy)


def _flags(union, gpu_semantics, exact):
    return ((FLAG_UNION if union else 0) | (FLAG_GPU_SEMANTICS if gpu_semantics else 0)
            | (FLAG_EXACT if exact else 0))


def exact_signs(v, dot=False):
    """Exact signs of A3 over rows (px,py,qx,qy,rx,ry), or of (U1-U0).(V1-V0) over rows
    (u1x,u1y,u0x,u0y,v1x,v1y,v0x,v0y) when dot."""
    v = np.ascontiguousarray(v, np.float64)
    n = v.shape[0]
    out = np.zeros(n, np.int32)
    lib().orc_exact_signs(_p(v), n, 1 if dot else 0, _p(out))
    return out


def clip_pair(P, Q, eps=1e-7, eps_clean=None, union=False, gpu_semantics=True, exact=False):
    P = np.ascontiguousarray(P, np.float64).reshape(-1)
    Q = np.ascontiguousarray(Q, np.float64).reshape(-1)
    flags = _flags(union, gpu_semantics, exact)
    lib().orc_clip_pair(_p(P), len(P) // 2, _p(Q), len(Q) // 2, eps,
                        eps if eps_clean is None else eps_clean, flags)
    return _collect()


def clip_multi(P_rings, Q_rings, eps=1e-7, eps_clean=None, union=False, gpu_semantics=True, exact=False):
    """Clip a pair of multi-component polygons (lists of open rings; holes by even-odd)."""
    P = np.ascontiguousarray(np.concatenate([np.asarray(r, np.float64).reshape(-1) for r in P_rings]))
    Q = np.ascontiguousarray(np.concatenate([np.asarray(r, np.float64).reshape(-1) for r in Q_rings]))
    sp = np.array([len(np.asarray(r).reshape(-1)) // 2 for r in P_rings], np.int32)
    sq = np.array([len(np.asarray(r).reshape(-1)) // 2 for r in Q_rings], np.int32)
    flags = _flags(union, gpu_semantics, exact)
    lib().orc_clip_multi(_p(P), _p(sp), len(sp), _p(Q), _p(sq), len(sq), eps,
                         eps if eps_clean is None else eps_clean, flags)
    return _collect()


INTERSECTION_FIELDS = ("xy_p", "xy_q", "alpha_p", "alpha_q", "label_p", "label_q", "neighbor_p", "neighbor_q")


def pair_intersections(P, Q, eps=1e-7, exact=False):
    """What the reference's calculateIntersections returns for P (not swapped) against Q:
    dict with status, n_p, n_q, invalid and, unless invalid, the merged rings (xy_*), keys
    (alpha_*), initial labels (label_*) and 1-based neighbours (neighbor_*)."""
    P = np.ascontiguousarray(P, np.float64).reshape(-1)
    Q = np.ascontiguousarray(Q, np.float64).reshape(-1)
    out3 = np.zeros(3, np.int64)
    st = lib().orc_pair_intersections(_p(P), len(P) // 2, _p(Q), len(Q) // 2, eps,
                                      FLAG_EXACT if exact else 0, _p(out3))
    r = {"status": int(st), "n_p": int(out3[0]), "n_q": int(out3[1]), "invalid": int(out3[2])}
    if r["invalid"]:
        return r
    np_, nq = r["n_p"], r["n_q"]
    arrs = [np.zeros(2 * np_), np.zeros(2 * nq)] + [np.zeros(n, np.int32) for n in (np_, nq) * 3]
    arrs = [arrs[0], arrs[1], arrs[2], arrs[3], arrs[4], arrs[5], arrs[6], arrs[7]]
    lib().orc_pair_intersections_copy(*[_p(a) for a in arrs])
    r.update(zip(INTERSECTION_FIELDS, arrs))
    return r


def clip_batch(base, overlay, pid, qid, eps=1e-7, eps_clean=None, union=False,
               gpu_semantics=True, exact=False):
    """Clip the listed (base, overlay) pairs with the reference's swap rule.  exact=True
    selects the exact-predicate mode (classification and orientation signs exact)."""
    pid = np.ascontiguousarray(pid, np.int32)
    qid = np.ascontiguousarray(qid, np.int32)
    flags = _flags(union, gpu_semantics, exact)
    lib().orc_clip_batch(_p(base.xy), _p(base.vnum), _p(base.vps),
                         _p(overlay.xy), _p(overlay.vnum), _p(overlay.vps),
                         _p(pid), _p(qid), len(pid), eps,
                         eps if eps_clean is None else eps_clean, flags)
    return _collect()


# ---------------------------------------------------------------- reference binary

def ref_available() -> bool:
    return os.path.exists(REF_BIN)


def write_pair_batch(path, pairs):
    with open(path, "wb") as f:
        f.write(struct.pack("<q", len(pairs)))
        for P, Q in pairs:
            P = np.ascontiguousarray(P, np.float64).reshape(-1, 2)
            Q = np.ascontiguousarray(Q, np.float64).reshape(-1, 2)
            f.write(struct.pack("<ii", len(P), len(Q)))
            f.write(P.tobytes())
            f.write(Q.tobytes())


def read_result_batch(path):
    data = open(path, "rb").read()
    off = 0
    (n,) = struct.unpack_from("<q", data, off)
    off += 8
    res = []
    for _ in range(n):
        (nc,) = struct.unpack_from("<i", data, off)
        off += 4
        comps = []
        for _ in range(nc):
            (nv,) = struct.unpack_from("<i", data, off)
            off += 4
            comps.append(np.frombuffer(data, np.float64, 2 * nv, off).reshape(-1, 2).copy())
            off += 16 * nv
        res.append(comps)
    return res


def ref_clip_pairs(pairs, union=False):
    """Run the reference's own sequential clipper (built from its sources) on pairs."""
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "in.bin")
        fout = os.path.join(td, "out.bin")
        write_pair_batch(fin, pairs)
        cmd = [REF_BIN, "batch", fin, fout] + (["union"] if union else [])
        subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
        return read_result_batch(fout)


def ref_clip_multi(pairs, union=False):
    """The reference's own sequential clipper on multi-component pairs: pairs is a list of
    (P rings, Q rings), each a list of open rings."""
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "in.bin")
        fout = os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            f.write(struct.pack("<q", len(pairs)))
            for Ps, Qs in pairs:
                for rings in (Ps, Qs):
                    f.write(struct.pack("<i", len(rings)))
                    f.write(np.array([len(np.asarray(r).reshape(-1, 2)) for r in rings], np.int32).tobytes())
                for rings in (Ps, Qs):
                    for r in rings:
                        f.write(np.ascontiguousarray(r, np.float64).reshape(-1).tobytes())
        cmd = [REF_BIN, "mbatch", fin, fout] + (["union"] if union else [])
        subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
        return read_result_batch(fout)


RING_FIELDS = ("x", "y", "alpha", "source", "inter", "label", "nb")


def ref_rings(pairs):
    """The reference's own merged vertex lists after computeIntersections plus the step-1
    labels, per pair: a (P list, Q list) tuple of dicts of arrays named RING_FIELDS."""
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "in.bin")
        fout = os.path.join(td, "out.bin")
        write_pair_batch(fin, pairs)
        subprocess.run([REF_BIN, "rings", fin, fout], check=True, stdout=subprocess.DEVNULL)
        data = open(fout, "rb").read()
    rec = np.dtype([("x", "<f8"), ("y", "<f8"), ("alpha", "<f8"), ("source", "<i4"), ("inter", "<i4"),
                    ("label", "<i4"), ("nb", "<i4")])
    off = 8
    out = []
    for _ in range(struct.unpack_from("<q", data, 0)[0]):
        n_p, n_q = struct.unpack_from("<ii", data, off)
        off += 8
        sides = []
        for n in (n_p, n_q):
            a = np.frombuffer(data, rec, n, off)
            off += n * rec.itemsize
            sides.append({f: a[f].copy() for f in RING_FIELDS})
        out.append(tuple(sides))
    return out


def ref_time_pairs(pairs, reps=1, union=False):
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "in.bin")
        write_pair_batch(fin, pairs)
        cmd = [REF_BIN, "time", fin, str(reps)] + (["union"] if union else [])
        out = subprocess.run(cmd, check=True, capture_output=True, text=True).stdout.split()
        return float(out[0]), int(out[1])


# ---------------------------------------------------------------- join

class JoinResult:
    pass


def _join_lib():
    L = lib()
    if not getattr(L, "_join_ready", False):
        vp, i64 = ctypes.c_void_p, ctypes.c_int64
        L.orc_join.argtypes = [vp, vp, vp, i64, vp, vp, vp, i64]
        L.orc_join.restype = i64
        L.orc_join_copy.argtypes = [vp] * 14
        L.orc_join_copy.restype = None
        L.orc_join_bruteforce.argtypes = [vp, vp, vp, i64, vp, vp, vp, i64, vp, vp, i64]
        L.orc_join_bruteforce.restype = i64
        L.orc_mbr.argtypes = [vp, vp, vp, i64, vp, vp]
        L.orc_mbr.restype = None
        L._join_ready = True
    return L


def mbr(layer):
    L = _join_lib()
    m = np.zeros(4 * layer.n_polys, np.float64)
    v = np.zeros(layer.n_polys, np.uint8)
    L.orc_mbr(_p(layer.xy), _p(layer.vnum), _p(layer.vps), layer.n_polys, _p(m), _p(v))
    return m.reshape(-1, 4), v


def join(base, overlay):
    L = _join_lib()
    K = L.orc_join(_p(base.xy), _p(base.vnum), _p(base.vps), base.n_polys,
                   _p(overlay.xy), _p(overlay.vnum), _p(overlay.vps), overlay.n_polys)
    r = JoinResult()
    r.b = np.zeros(K, np.int32)
    r.o = np.zeros(K, np.int32)
    r.cmbr = np.zeros(4 * K, np.float64)
    r.pip_type = np.zeros(K, np.int8)
    r.pip_flag = np.zeros(K, np.int8)
    r.join_flag = np.zeros(K, np.int8)
    r.bE = np.zeros(K, np.int32)
    r.oE = np.zeros(K, np.int32)
    r.seg_flag = np.zeros(K, np.int8)
    r.clip = np.zeros(K, np.int8)
    r.mbr_b = np.zeros(4 * base.n_polys, np.float64)
    r.valid_b = np.zeros(base.n_polys, np.uint8)
    r.mbr_o = np.zeros(4 * overlay.n_polys, np.float64)
    r.valid_o = np.zeros(overlay.n_polys, np.uint8)
    L.orc_join_copy(_p(r.b), _p(r.o), _p(r.cmbr), _p(r.pip_type), _p(r.pip_flag),
                    _p(r.join_flag), _p(r.bE), _p(r.oE), _p(r.seg_flag), _p(r.clip),
                    _p(r.mbr_b), _p(r.valid_b), _p(r.mbr_o), _p(r.valid_o))
    r.cmbr = r.cmbr.reshape(-1, 4)
    return r


def join_bruteforce(base, overlay):
    L = _join_lib()
    cap = 1 << 22
    while True:
        ob = np.zeros(cap, np.int32)
        oo = np.zeros(cap, np.int32)
        k = L.orc_join_bruteforce(_p(base.xy), _p(base.vnum), _p(base.vps), base.n_polys,
                                  _p(overlay.xy), _p(overlay.vnum), _p(overlay.vps),
                                  overlay.n_polys, _p(ob), _p(oo), cap)
        if k <= cap:
            return ob[:k].copy(), oo[:k].copy()
        cap = int(k)
