"""Python front end of libgcmfgh.so (the C ABI in include/gcmfgh.h).

The engine itself is C++/CUDA; this module only moves arrays across the C ABI with
ctypes.  Device memory comes from torch tensors on the context's device.  Nothing here
computes results: if the shared library or the GPU is missing, the calls raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import synth  # noqa: F401  (re-exported for harness code)

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libgcmfgh.so")

# gcmf_join_field
JOIN_FIELDS = {
    "b": (0, np.int32), "o": (1, np.int32), "cmbr": (2, np.float64), "pip_type": (3, np.int8),
    "pip_flag": (4, np.int8), "join_flag": (5, np.int8), "bE": (6, np.int32), "oE": (7, np.int32),
    "seg_flag": (8, np.int8), "clip": (9, np.int8), "clip_b": (10, np.int32), "clip_o": (11, np.int32),
    "mbr_b": (12, np.float64), "mbr_o": (13, np.float64), "valid_b": (14, np.uint8),
    "valid_o": (15, np.uint8),
}
# gh_clip_field
CLIP_FIELDS = {
    "status": (0, np.int32), "ncomp": (1, np.int32), "comp_off": (2, np.int64),
    "count1": (3, np.int64), "comp_size": (4, np.int32), "vert_off": (5, np.int64),
    "xy": (6, np.float64), "swapped": (7, np.int32),
}


class GcmfghError(RuntimeError):
    pass


def launch_count() -> int:
    """Kernels launched by libgcmfgh.so in this process so far."""
    return int(lib().gcmfgh_launch_count())


class Layer(ctypes.Structure):
    _fields_ = [("coords", ctypes.c_void_p), ("vnum", ctypes.c_void_p), ("vps", ctypes.c_void_p),
                ("n_polys", ctypes.c_int64), ("n_vertices", ctypes.c_int64)]


class Tuning(ctypes.Structure):
    _fields_ = [("bin_grid", ctypes.c_int64), ("tile_label", ctypes.c_int64), ("mid_label", ctypes.c_int64),
                ("big_label", ctypes.c_int64), ("wide_label", ctypes.c_int64), ("pairs_log2", ctypes.c_int),
                ("verts_log2", ctypes.c_int), ("exact", ctypes.c_int), ("ms_default", ctypes.c_double),
                ("ms_tuned", ctypes.c_double), ("configs_timed", ctypes.c_int)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class JoinInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in
                ("n_pairs", "n_pip_candidates", "n_within", "n_cmf", "n_seg", "n_clip")]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


class ClipInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in
                ("n_pairs", "n_components", "n_vertices", "n_invalid", "n_disjoint", "n_error",
                 "n_records", "n_ring_vertices")]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


class Intersections(ctypes.Structure):
    _fields_ = [("n_p", ctypes.c_int64), ("n_q", ctypes.c_int64), ("invalid", ctypes.c_int32),
                ("xy_p", ctypes.c_void_p), ("xy_q", ctypes.c_void_p),
                ("alpha_p", ctypes.c_void_p), ("alpha_q", ctypes.c_void_p),
                ("label_p", ctypes.c_void_p), ("label_q", ctypes.c_void_p),
                ("neighbor_p", ctypes.c_void_p), ("neighbor_q", ctypes.c_void_p)]


class ServeOptions(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("workers", ctypes.c_int),
                ("max_batch_queries", ctypes.c_int64), ("max_batch_vertices", ctypes.c_int64),
                ("reserve_bytes", ctypes.c_int64), ("bytes_per_vertex", ctypes.c_int64),
                ("eps", ctypes.c_double), ("eps_clean", ctypes.c_double),
                ("union_mode", ctypes.c_int), ("exact", ctypes.c_int)]


class ServeResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32)] + [(n, ctypes.c_int64) for n in
                ("n_hits", "n_components", "n_vertices", "n_candidates", "arrival_ns", "admitted_ns",
                 "done_ns", "batch_id", "batch_queries")]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise GcmfghError(f"{LIB_PATH} is not built (run __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        vp, i32, i64, d = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
        P = ctypes.POINTER
        L.gcmfgh_create.argtypes = [ctypes.c_int, P(vp)]
        L.gcmfgh_destroy.argtypes = [vp]
        L.gcmfgh_set_stream.argtypes = [vp, vp]
        L.gcmfgh_set_params.argtypes = [vp, d, d, ctypes.c_int]
        L.gcmfgh_set_precision.argtypes = [vp, ctypes.c_int]
        L.gcmfgh_status_string.argtypes = [ctypes.c_int]
        L.gcmfgh_status_string.restype = ctypes.c_char_p
        L.gcmfgh_last_device_error.argtypes = [vp]
        L.gcmf_join.argtypes = [vp, P(Layer), P(Layer), P(JoinInfo)]
        L.gcmf_join_get.argtypes = [vp, ctypes.c_int, vp, i64, ctypes.c_int, P(i64)]
        L.gcmf_join_ptr.argtypes = [vp, ctypes.c_int, P(vp), P(i64)]
        L.gh_clip_batch.argtypes = [vp, P(Layer), P(Layer), vp, vp, i64, P(ClipInfo)]
        L.gh_clip_joined.argtypes = [vp, P(Layer), P(Layer), P(ClipInfo)]
        L.gcmfgh_autotune_joined.argtypes = [vp, P(Layer), P(Layer), P(Tuning)]
        L.gcmfgh_tuning_for.argtypes = [vp, P(Layer), P(Layer), i64, P(Tuning)]
        L.gh_clip_batch_host_ids.argtypes = [vp, P(Layer), P(Layer), vp, vp, i64, P(ClipInfo)]
        L.gh_clip_get.argtypes = [vp, ctypes.c_int, vp, i64, ctypes.c_int, P(i64)]
        L.gh_clip_ptr.argtypes = [vp, ctypes.c_int, P(vp), P(i64)]
        L.gh_clip_pair.argtypes = [vp, vp, i32, vp, i32, P(ClipInfo)]
        L.gh_clip_multi.argtypes = [vp, vp, vp, i32, vp, vp, i32, P(ClipInfo)]
        L.gh_clip_multi_batch.argtypes = [vp, i64, vp, vp, vp, vp, vp, vp, P(ClipInfo)]
        L.gh_calculate_intersections.argtypes = [vp, P(Layer), i32, P(Layer), i32, P(Intersections)]
        L.gh_free_intersections.argtypes = [P(Intersections)]
        L.gh_free_intersections.restype = None
        L.gcmfgh_join_clip_host.argtypes = [vp, P(Layer), P(Layer), P(JoinInfo), P(ClipInfo)]
        L.gcmfgh_exclusive_scan_i32.argtypes = [vp, vp, vp, i64, P(i64)]
        L.gcmfgh_radix_sort_u64.argtypes = [vp, vp, vp, i64, ctypes.c_int]
        L.gcmfgh_launch_count.argtypes = []
        L.gcmfgh_launch_count.restype = ctypes.c_ulonglong
        L.gcmfgh_set_tuning.argtypes = [vp, ctypes.c_int, i64]
        L.gcmfgh_set_timing.argtypes = [vp, ctypes.c_int]
        L.gcmfgh_get_timing.argtypes = [vp, ctypes.c_int, P(ctypes.c_float), P(ctypes.c_char_p),
                                        ctypes.c_int]
        L.gcmfgh_get_timing.restype = ctypes.c_int
        L.gcmfgh_serve_default_options.argtypes = [P(ServeOptions)]
        L.gcmfgh_serve_open.argtypes = [P(Layer), P(ServeOptions), P(vp)]
        L.gcmfgh_serve_submit.argtypes = [vp, vp, i32, i64, P(ctypes.c_uint64)]
        L.gcmfgh_serve_poll.argtypes = [vp, ctypes.c_uint64, P(ServeResult)]
        L.gcmfgh_serve_wait.argtypes = [vp, ctypes.c_uint64, i64, P(ServeResult)]
        L.gcmfgh_serve_take.argtypes = [vp, ctypes.c_uint64, vp, vp, vp, vp, vp]
        L.gcmfgh_serve_stats.argtypes = [vp, P(i64), P(i64), P(i64)]
        L.gcmfgh_serve_close.argtypes = [vp]
        L.gcmfgh_serve_phases.argtypes = [vp, vp, vp]
        _lib = L
    return _lib


def _check(st):
    if st != 0:
        raise GcmfghError(f"gcmfgh: {lib().gcmfgh_status_string(st).decode()} ({st})")


def _np_ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


class DeviceLayer:
    """A layer resident on the GPU (torch tensors) plus its C view."""

    def __init__(self, layer, device="cuda:0"):
        import torch
        self.layer = layer
        self.xy = torch.from_numpy(layer.xy).to(device)
        self.vnum = torch.from_numpy(layer.vnum).to(device)
        self.vps = torch.from_numpy(layer.vps).to(device)
        self.c = Layer(self.xy.data_ptr(), self.vnum.data_ptr(), self.vps.data_ptr(),
                       layer.n_polys, layer.n_vertices)


def _device_layer_from_tensors(xy, vnum, vps):
    """DeviceLayer over device tensors already in the layer layout (xy f64 interleaved
    with closing vertices, vnum i32, vps i64 inclusive)."""
    d = DeviceLayer.__new__(DeviceLayer)
    d.layer = None
    d.xy, d.vnum, d.vps = xy.contiguous(), vnum.contiguous(), vps.contiguous()
    n = int(d.vnum.numel())
    nv = int(d.vps[-1].item()) if n else 0
    d.c = Layer(d.xy.data_ptr(), d.vnum.data_ptr(), d.vps.data_ptr(), n, nv)
    return d


DeviceLayer.from_tensors = staticmethod(_device_layer_from_tensors)


def host_layer(layer):
    """C view of a host (numpy) layer for the host-buffer entry point."""
    return Layer(layer.xy.ctypes.data, layer.vnum.ctypes.data, layer.vps.ctypes.data,
                 layer.n_polys, layer.n_vertices)


class ClipResult:
    """Per-pair status and result components, host copies (same shape as the oracle's)."""

    def __init__(self, status, ncomp, count1, comp_size, xy, swapped):
        self.status = status
        self.ncomp = ncomp
        self.count1 = count1
        self.comp_size = comp_size
        self.xy = xy
        self.swapped = swapped
        self.comp_off = np.concatenate([[0], np.cumsum(comp_size, dtype=np.int64)])
        self.pair_comp_off = np.concatenate([[0], np.cumsum(ncomp, dtype=np.int64)])

    def components(self, k):
        out = []
        for c in range(self.pair_comp_off[k], self.pair_comp_off[k + 1]):
            a, b = self.comp_off[c], self.comp_off[c + 1]
            out.append(self.xy[2 * a:2 * b].reshape(-1, 2))
        return out


class Engine:
    """One gcmfgh context on one GPU."""

    def __init__(self, device=0, eps=1e-7, eps_clean=None, union=False):
        self.device = device
        h = ctypes.c_void_p()
        _check(lib().gcmfgh_create(device, ctypes.byref(h)))
        self.h = h
        self.set_params(eps, eps if eps_clean is None else eps_clean, union)

    def close(self):
        if self.h:
            lib().gcmfgh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, eps=1e-7, eps_clean=1e-7, union=False):
        _check(lib().gcmfgh_set_params(self.h, eps, eps_clean, 1 if union else 0))

    def set_precision(self, exact=False):
        """exact=True: exact orientation/classification signs (eps unused there)."""
        _check(lib().gcmfgh_set_precision(self.h, 1 if exact else 0))

    def set_stream(self, stream_ptr):
        _check(lib().gcmfgh_set_stream(self.h, ctypes.c_void_p(stream_ptr)))

    def last_device_error(self):
        return lib().gcmfgh_last_device_error(self.h)

    def set_tuning(self, bin_grid=None, big_label=None, mid_label=None, tile_label=None, wide_label=None,
                   f32_filter=None, fused_emit=None, record_hint=None, join_sweep=None,
                   sweep_two_pass=None):
        """Work-distribution thresholds, the join's FP32 prefilters, the one-pass record
        count + emit and its capacity hint (results depend on none of them)."""
        if f32_filter is not None:      # bit 0: MBR y prefilter, bit 1: edge prefilter
            _check(lib().gcmfgh_set_tuning(self.h, 5, int(f32_filter)))
        if fused_emit is not None:
            _check(lib().gcmfgh_set_tuning(self.h, 6, int(fused_emit)))
        if record_hint is not None:     # 0: the last clip's record count
            _check(lib().gcmfgh_set_tuning(self.h, 7, int(record_hint)))
        if join_sweep is not None:      # MBR candidates by the sort-sweep instead of the grid probe
            _check(lib().gcmfgh_set_tuning(self.h, 8, 1 if join_sweep else 0))
        if sweep_two_pass is not None:  # the sweep's count and emit as two passes
            _check(lib().gcmfgh_set_tuning(self.h, 9, 1 if sweep_two_pass else 0))
        if bin_grid is not None:
            _check(lib().gcmfgh_set_tuning(self.h, 0, int(bin_grid)))
        if big_label is not None:
            _check(lib().gcmfgh_set_tuning(self.h, 1, int(big_label)))
        if mid_label is not None:
            _check(lib().gcmfgh_set_tuning(self.h, 2, int(mid_label)))
        if tile_label is not None:
            _check(lib().gcmfgh_set_tuning(self.h, 3, int(tile_label)))
        if wide_label is not None:
            _check(lib().gcmfgh_set_tuning(self.h, 4, int(wide_label)))

    def autotune_joined(self, dbase: DeviceLayer, dovl: DeviceLayer):
        """Times the last join's clip set under candidate work-distribution thresholds and
        records the fastest for this workload's signature (gcmfgh_autotune_joined)."""
        t = Tuning()
        _check(lib().gcmfgh_autotune_joined(self.h, ctypes.byref(dbase.c), ctypes.byref(dovl.c), ctypes.byref(t)))
        return t.as_dict()

    def tuning_for(self, dbase: DeviceLayer, dovl: DeviceLayer, n_pairs):
        t = Tuning()
        _check(lib().gcmfgh_tuning_for(self.h, ctypes.byref(dbase.c), ctypes.byref(dovl.c), int(n_pairs),
                                       ctypes.byref(t)))
        return t.as_dict()

    def set_timing(self, on=True):
        _check(lib().gcmfgh_set_timing(self.h, 1 if on else 0))

    def timing(self, which):
        """[(stage, ms)] of the last join (which=0) or clip (which=1)."""
        ms = (ctypes.c_float * 32)()
        names = (ctypes.c_char_p * 32)()
        n = lib().gcmfgh_get_timing(self.h, which, ms, names, 32)
        return [(names[i].decode(), float(ms[i])) for i in range(max(n, 0))]

    # ---- join
    def join(self, dbase: DeviceLayer, dovl: DeviceLayer):
        info = JoinInfo()
        _check(lib().gcmf_join(self.h, ctypes.byref(dbase.c), ctypes.byref(dovl.c), ctypes.byref(info)))
        return info.as_dict()

    def _get(self, getter, fields, name):
        fid, dt = fields[name]
        nbytes = ctypes.c_int64()
        _check(getter(self.h, fid, None, 0, 0, ctypes.byref(nbytes)))
        out = np.empty(nbytes.value // np.dtype(dt).itemsize, dtype=dt)
        _check(getter(self.h, fid, _np_ptr(out), nbytes.value, 0, ctypes.byref(nbytes)))
        return out

    def join_field(self, name):
        return self._get(lib().gcmf_join_get, JOIN_FIELDS, name)

    def clip_field(self, name):
        return self._get(lib().gh_clip_get, CLIP_FIELDS, name)

    def clip_ptr(self, name):
        fid, _ = CLIP_FIELDS[name]
        p = ctypes.c_void_p()
        n = ctypes.c_int64()
        _check(lib().gh_clip_ptr(self.h, fid, ctypes.byref(p), ctypes.byref(n)))
        return p.value, n.value

    # ---- clip
    def clip_batch(self, dbase: DeviceLayer, dovl: DeviceLayer, pid, qid):
        import torch
        dev = dbase.xy.device
        if isinstance(pid, torch.Tensor):
            p = pid.to(device=dev, dtype=torch.int32).contiguous()
            q = qid.to(device=dev, dtype=torch.int32).contiguous()
        else:
            p = torch.as_tensor(np.ascontiguousarray(pid, np.int32)).to(dev)
            q = torch.as_tensor(np.ascontiguousarray(qid, np.int32)).to(dev)
        info = ClipInfo()
        _check(lib().gh_clip_batch(self.h, ctypes.byref(dbase.c), ctypes.byref(dovl.c),
                                   ctypes.c_void_p(p.data_ptr()), ctypes.c_void_p(q.data_ptr()),
                                   len(pid), ctypes.byref(info)))
        return info.as_dict()

    def clip_joined(self, dbase: DeviceLayer, dovl: DeviceLayer):
        info = ClipInfo()
        _check(lib().gh_clip_joined(self.h, ctypes.byref(dbase.c), ctypes.byref(dovl.c), ctypes.byref(info)))
        return info.as_dict()

    def clip_pair(self, P, Q):
        P = np.ascontiguousarray(P, np.float64).reshape(-1)
        Q = np.ascontiguousarray(Q, np.float64).reshape(-1)
        info = ClipInfo()
        _check(lib().gh_clip_pair(self.h, _np_ptr(P), len(P) // 2, _np_ptr(Q), len(Q) // 2,
                                  ctypes.byref(info)))
        return info.as_dict()

    def clip_multi(self, P_rings, Q_rings):
        """Clip one pair of multi-component polygons (lists of open rings, holes by
        even-odd); read the result with clip_result()."""
        P = np.ascontiguousarray(np.concatenate([np.asarray(r, np.float64).reshape(-1) for r in P_rings]))
        Q = np.ascontiguousarray(np.concatenate([np.asarray(r, np.float64).reshape(-1) for r in Q_rings]))
        sp = np.array([len(np.asarray(r).reshape(-1)) // 2 for r in P_rings], np.int32)
        sq = np.array([len(np.asarray(r).reshape(-1)) // 2 for r in Q_rings], np.int32)
        info = ClipInfo()
        _check(lib().gh_clip_multi(self.h, _np_ptr(P), _np_ptr(sp), len(sp), _np_ptr(Q), _np_ptr(sq), len(sq),
                                   ctypes.byref(info)))
        return info.as_dict()

    def clip_multi_batch(self, pairs):
        """Clip a batch of multi-component polygon pairs, [(P_rings, Q_rings), ...], in one
        call (gh_clip_multi_batch); read the results with clip_result()."""
        def side(idx):
            rings = [np.asarray(r, np.float64).reshape(-1) for pq in pairs for r in pq[idx]]
            xy = np.ascontiguousarray(np.concatenate(rings))
            sizes = np.array([len(r) // 2 for r in rings], np.int32)
            counts = np.array([len(pq[idx]) for pq in pairs], np.int32)
            return xy, sizes, counts
        P, sp, cp = side(0)
        Q, sq, cq = side(1)
        info = ClipInfo()
        _check(lib().gh_clip_multi_batch(self.h, len(pairs), _np_ptr(P), _np_ptr(sp), _np_ptr(cp), _np_ptr(Q),
                                         _np_ptr(sq), _np_ptr(cq), ctypes.byref(info)))
        return info.as_dict()

    def calculate_intersections(self, p_layer: DeviceLayer, p_id, q_layer: DeviceLayer, q_id):
        """The reference's calculateIntersections for polygon p_id of p_layer (P, not swapped)
        against polygon q_id of q_layer: dict with n_p, n_q, invalid and, unless invalid,
        numpy copies of the merged rings (xy_*), keys (alpha_*), initial labels (label_*)
        and 1-based neighbours (neighbor_*)."""
        x = Intersections()
        _check(lib().gh_calculate_intersections(self.h, ctypes.byref(p_layer.c), int(p_id), ctypes.byref(q_layer.c),
                                                int(q_id), ctypes.byref(x)))
        try:
            r = {"n_p": int(x.n_p), "n_q": int(x.n_q), "invalid": int(x.invalid)}
            if not x.invalid:
                for name, n, ct, dt in (("xy_p", 2 * x.n_p, ctypes.c_double, np.float64),
                                        ("xy_q", 2 * x.n_q, ctypes.c_double, np.float64),
                                        ("alpha_p", x.n_p, ctypes.c_int32, np.int32),
                                        ("alpha_q", x.n_q, ctypes.c_int32, np.int32),
                                        ("label_p", x.n_p, ctypes.c_int32, np.int32),
                                        ("label_q", x.n_q, ctypes.c_int32, np.int32),
                                        ("neighbor_p", x.n_p, ctypes.c_int32, np.int32),
                                        ("neighbor_q", x.n_q, ctypes.c_int32, np.int32)):
                    ptr = getattr(x, name)
                    r[name] = (np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ct)), shape=(n,)).astype(dt)
                               if n > 0 else np.zeros(0, dt))
            return r
        finally:
            lib().gh_free_intersections(ctypes.byref(x))

    def clip_result_pairs(self, pairs):
        """Host copies of the results of the listed pairs only (the rest stays on the
        device): (status, [components per pair])."""
        import torch
        dev = torch.device("cuda", torch.cuda.current_device())

        def field(name):
            fid, dt = CLIP_FIELDS[name]
            p = ctypes.c_void_p()
            n = ctypes.c_int64()
            _check(lib().gh_clip_ptr(self.h, fid, ctypes.byref(p), ctypes.byref(n)))
            out = torch.empty(max(n.value, 1), dtype={np.int32: torch.int32, np.int64: torch.int64,
                                                      np.float64: torch.float64}[dt], device=dev)
            nb = ctypes.c_int64()
            _check(lib().gh_clip_get(self.h, fid, ctypes.c_void_p(out.data_ptr()),
                                     out.numel() * out.element_size(), 1, ctypes.byref(nb)))
            return out[:n.value]

        pairs = np.asarray(pairs, np.int64)
        status, ncomp = field("status"), field("ncomp")
        coff, voff, csz, xy = field("comp_off"), field("vert_off"), field("comp_size"), field("xy")
        sel = torch.as_tensor(pairs, device=dev)
        st = status[sel].cpu().numpy()
        nc = ncomp[sel].cpu().numpy()
        c0 = coff[sel].cpu().numpy()
        v0 = voff[sel].cpu().numpy()
        comps = []
        for k in range(len(pairs)):
            sizes = csz[int(c0[k]):int(c0[k]) + int(nc[k])].cpu().numpy() if nc[k] else np.zeros(0, np.int32)
            n = int(sizes.sum())
            v = xy[2 * int(v0[k]):2 * (int(v0[k]) + n)].cpu().numpy().reshape(-1, 2)
            comps.append(np.split(v, np.cumsum(sizes)[:-1]) if n else [])
        return st, comps

    def clip_result(self):
        return ClipResult(self.clip_field("status"), self.clip_field("ncomp"), self.clip_field("count1"),
                          self.clip_field("comp_size"), self.clip_field("xy"), self.clip_field("swapped"))

    # ---- primitives (device tensors)
    def exclusive_scan_i32(self, d_in):
        import torch
        out = torch.empty(d_in.numel(), dtype=torch.int64, device=d_in.device)
        tot = ctypes.c_int64()
        _check(lib().gcmfgh_exclusive_scan_i32(self.h, ctypes.c_void_p(d_in.data_ptr()),
                                               ctypes.c_void_p(out.data_ptr()), d_in.numel(),
                                               ctypes.byref(tot)))
        return out, tot.value

    def radix_sort_u64(self, d_keys, d_vals, key_bits=64):
        """Sorts int64-typed tensors holding u64 keys in place (unsigned order)."""
        _check(lib().gcmfgh_radix_sort_u64(self.h, ctypes.c_void_p(d_keys.data_ptr()),
                                           ctypes.c_void_p(d_vals.data_ptr()), d_keys.numel(), key_bits))

    # ---- end to end from host buffers
    def join_clip_host(self, base, ovl):
        jb, jo = host_layer(base), host_layer(ovl)
        ji, ci = JoinInfo(), ClipInfo()
        _check(lib().gcmfgh_join_clip_host(self.h, ctypes.byref(jb), ctypes.byref(jo), ctypes.byref(ji),
                                           ctypes.byref(ci)))
        return ji.as_dict(), ci.as_dict()


class QueryResult:
    """One served query: per hit the resident polygon id, clip status and components."""

    def __init__(self, info, hit_ids, hit_status, hit_ncomp, comp_size, xy):
        self.info = info
        self.hit_ids, self.hit_status, self.hit_ncomp = hit_ids, hit_status, hit_ncomp
        self.comp_size, self.xy = comp_size, xy

    def latency_ns(self):
        return self.info["done_ns"] - self.info["arrival_ns"]


class Server:
    """Continuous-batching join+clip server over a resident (host numpy) layer."""

    def __init__(self, resident, device=0, workers=2, max_batch_queries=4096,
                 max_batch_vertices=1 << 22, reserve_bytes=2 << 30, bytes_per_vertex=4096,
                 eps=1e-7, eps_clean=1e-7, union=False, exact=False):
        o = ServeOptions()
        _check(lib().gcmfgh_serve_default_options(ctypes.byref(o)))
        o.device, o.workers = device, workers
        o.max_batch_queries, o.max_batch_vertices = max_batch_queries, max_batch_vertices
        o.reserve_bytes, o.bytes_per_vertex = reserve_bytes, bytes_per_vertex
        o.eps, o.eps_clean, o.union_mode, o.exact = eps, eps_clean, int(union), int(exact)
        self._resident = resident
        self.h = ctypes.c_void_p()
        L = host_layer(resident)
        _check(lib().gcmfgh_serve_open(ctypes.byref(L), ctypes.byref(o), ctypes.byref(self.h)))

    def submit(self, ring, arrival_ns=0):
        r = np.ascontiguousarray(ring, np.float64).reshape(-1)
        t = ctypes.c_uint64()
        _check(lib().gcmfgh_serve_submit(self.h, _np_ptr(r), len(r) // 2, int(arrival_ns), ctypes.byref(t)))
        return t.value

    def poll(self, ticket):
        info = ServeResult()
        st = lib().gcmfgh_serve_poll(self.h, ticket, ctypes.byref(info))
        if st == 5:
            return None
        _check(st)
        return info.as_dict()

    def wait(self, ticket, timeout_ms=-1):
        info = ServeResult()
        st = lib().gcmfgh_serve_wait(self.h, ticket, int(timeout_ms), ctypes.byref(info))
        if st == 5:
            return None
        _check(st)
        return info.as_dict()

    def take(self, ticket, info):
        nh, nc, nv = info["n_hits"], info["n_components"], info["n_vertices"]
        ids, hst, hnc = (np.zeros(nh, np.int32) for _ in range(3))
        csz, xy = np.zeros(nc, np.int32), np.zeros(2 * nv, np.float64)
        _check(lib().gcmfgh_serve_take(self.h, ticket, _np_ptr(ids), _np_ptr(hst), _np_ptr(hnc),
                                       _np_ptr(csz), _np_ptr(xy)))
        return QueryResult(info, ids, hst, hnc, csz, xy)

    def result(self, ticket, timeout_ms=-1):
        info = self.wait(ticket, timeout_ms)
        if info is None:
            raise GcmfghError("query not finished within the timeout")
        return self.take(ticket, info)

    def stats(self):
        b, q, p = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _check(lib().gcmfgh_serve_stats(self.h, ctypes.byref(b), ctypes.byref(q), ctypes.byref(p)))
        return {"batches": b.value, "queries": q.value, "peak_batch": p.value}

    def phases(self):
        """Per-phase serving time (ms, summed over batches) and work totals."""
        ms = (ctypes.c_double * 7)()
        work = (ctypes.c_int64 * 4)()
        _check(lib().gcmfgh_serve_phases(self.h, ms, work))
        names = ("host_stage", "h2d", "candidates", "join_J3_J6", "clip", "d2h", "host_split")
        return ({n: ms[i] for i, n in enumerate(names)},
                dict(zip(("query_vertices", "pairs", "ring_vertices", "result_vertices"), list(work))))

    def close(self):
        if self.h:
            _check(lib().gcmfgh_serve_close(self.h))
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class TextLayer(ctypes.Structure):
    _fields_ = [("coords", ctypes.c_void_p), ("vnum", ctypes.c_void_p), ("vps", ctypes.c_void_p),
                ("ids", ctypes.c_void_p), ("n_polys", ctypes.c_int64), ("n_vertices", ctypes.c_int64)]


def read_text_layer(path, threads=0):
    """Parses a GCMF text layer file with the engine's parallel reader; returns
    (synth.Layer, ids)."""
    L = lib()
    L.gcmfgh_read_text_layer.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(TextLayer)]
    L.gcmfgh_free_text_layer.argtypes = [ctypes.POINTER(TextLayer)]
    L.gcmfgh_free_text_layer.restype = None
    t = TextLayer()
    _check(L.gcmfgh_read_text_layer(os.fsencode(path), int(threads), ctypes.byref(t)))
    try:
        n, nv = t.n_polys, t.n_vertices
        xy = np.ctypeslib.as_array(ctypes.cast(t.coords, ctypes.POINTER(ctypes.c_double)), (2 * max(nv, 1),))[:2 * nv].copy()
        vnum = np.ctypeslib.as_array(ctypes.cast(t.vnum, ctypes.POINTER(ctypes.c_int32)), (max(n, 1),))[:n].copy()
        ids = np.ctypeslib.as_array(ctypes.cast(t.ids, ctypes.POINTER(ctypes.c_int64)), (max(n, 1),))[:n].copy()
    finally:
        L.gcmfgh_free_text_layer(ctypes.byref(t))
    return synth.Layer(xy, vnum), ids


def write_text_layer(path, layer):
    """Writes a (host) layer in the GCMF text format."""
    L = lib()
    L.gcmfgh_write_text_layer.argtypes = [ctypes.c_char_p, ctypes.POINTER(Layer)]
    h = host_layer(layer)
    _check(L.gcmfgh_write_text_layer(os.fsencode(path), ctypes.byref(h)))
