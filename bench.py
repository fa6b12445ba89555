#!/usr/bin/env python
"""Join+clip polygon pairs/s on the batched spatial-join workload.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Workload (one step): the GCMF join of two layers of 200,000 FP64 star polygons (vertex
counts floor(Pareto(1.5, 4)) capped at 100,000; centres from a 64-component Gaussian
mixture over [0,1e5]^2, sigma 2,000; base radius log-normal(ln 50, 0.7); seed 2 on rank
0, 2+r on rank r), followed by the Greiner-Hormann clip of every pair in the clip set.
The unit is one clipped polygon pair.  Under torchrun every rank processes its own
instance (weak scaling, no data-path collective); value = all ranks' pairs / the
slowest rank's step time.

--impl reference times the reference's CPU path on the host cores instead: the GH clip by
the reference's own sequential clipper built from its sources (oracle/_ref), the join by
the oracle's restatement of its candidate/containment/edge-filter/refine stages, on a
bounded sample of base polygons per step.
"""
import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gcmf-gh_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402

METRIC = "join+clip polygon pairs/s at FP64-oracle accuracy"
WORKLOAD = ("batched_join: 200000 x 200000 FP64 star polygons, Pareto(1.5, min 4) vertices "
            "capped 1e5, 64-component GMM centres over [0,1e5]^2 (sigma 2000), base radius "
            "lognormal(ln 50, 0.7); GCMF join then GH clip of the clip set")
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--sample-bases", type=int, default=0,
                    help="reference arm: base polygons per step sample (0: auto)")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving latency section")
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the host-core reference sample")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


# ----------------------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        self.f.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------- roofline

def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def stage_bytes(stage, ji, ci, nb, no, vb, vo, cand_vertices=0):
    """Algorithmic bytes of one stage (reads of what it must read once + writes of what it
    must produce), from the step's counts.  cand_vertices is the sum over candidate pairs
    of both polygons' vertex counts: the common-MBR filter reads every edge of both
    polygons of each candidate once."""
    K, C = ji["n_pairs"], ci["n_pairs"]
    ring, out_v, recs = ci["n_ring_vertices"], ci["n_vertices"], ci["n_records"]
    table = {
        # merged P and Q rings read once (x, y), result vertices written, pair status
        "clip:label+trace": 16 * ring + 16 * out_v + 8 * C,
        # records read, merged rings written (x, y + neighbour link)
        "clip:fill+link": 33 * recs + 20 * ring,
        "clip:count": 16 * ring + 8 * C,
        "clip:emit": 16 * ring + 33 * recs,
        "join:mbr+sort": 16 * (vb + vo) + 40 * (nb + no),
        "join:sweep-count": 36 * (nb + no),
        "join:sweep-emit+sort": 36 * (nb + no) + 16 * K,
        "join:cmf": 16 * cand_vertices + 40 * K,
    }
    return table.get(stage)


def traffic_from_profiles(stage):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    v = d.get(stage)
    return None if v is None else float(v.get("dram_bytes_per_launch"))


# ----------------------------------------------------------------------------- CPU baseline

def swap_rings(base, ovl, b, o):
    """The GCMF-GH swap rule (GH-CUDA/ghcuda.cpp:64-91): the ring with more vertices is P."""
    P, Q = base.ring(b), ovl.ring(o)
    return (Q, P) if len(P) < len(Q) else (P, Q)


def reference_cpu_sample(base, ovl, n_bases, seed, max_procs=None):
    """One bounded sample of the workload on the host: every join candidate of n_bases
    randomly chosen base polygons against the whole overlay layer (oracle restatement of
    the reference's join stages), then the reference's own sequential GH clipper on the
    sample's clip set, in parallel worker processes over the host cores.
    Returns (pairs, seconds, cores)."""
    import pyoracle
    from gcmfgh import synth
    rng = np.random.default_rng(seed)
    ids = np.sort(rng.choice(base.n_polys, size=min(n_bases, base.n_polys), replace=False))
    sub = synth.Layer.from_rings([base.ring(int(i)) for i in ids])
    t0 = time.perf_counter()
    jr = pyoracle.join(sub, ovl)
    t_join = time.perf_counter() - t0
    sel = np.nonzero(jr.clip)[0]
    pairs = [swap_rings(sub, ovl, int(jr.b[k]), int(jr.o[k])) for k in sel]
    cores = max_procs or os.cpu_count() or 1
    cores = max(1, min(cores, len(pairs) // 64 or 1))
    chunks = [pairs[i::cores] for i in range(cores)]
    with tempfile.TemporaryDirectory() as td:
        procs = []
        for i, ch in enumerate(chunks):
            fn = os.path.join(td, f"c{i}.bin")
            pyoracle.write_pair_batch(fn, ch)
            procs.append(fn)
        t1 = time.perf_counter()
        running = [subprocess.Popen([pyoracle.REF_BIN, "time", fn, "1"], stdout=subprocess.PIPE, text=True)
                   for fn in procs]
        for p in running:
            p.communicate()
        t_clip = time.perf_counter() - t1
    return len(pairs), t_join + t_clip, cores


def run_reference(args, rank, world):
    if rank != 0:
        return
    import pyoracle
    from gcmfgh import synth
    if not pyoracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent at build time)"}))
        return
    pyoracle.lib()
    base, ovl = synth.batched_join(seed=2)
    nb = args.sample_bases or 20000
    for i in range(args.warmup):
        reference_cpu_sample(base, ovl, max(nb // 10, 100), 100 + i)
    pairs, secs = 0, 0.0
    cores = 1
    for i in range(args.steps):
        p, s, cores = reference_cpu_sample(base, ovl, nb, 1000 + i)
        pairs += p
        secs += s
    v = pairs / secs
    line = {
        "metric": METRIC, "value": v, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": WORKLOAD, "sample_bases_per_step": nb},
        "cpu_baseline": {"value": v, "unit": "pairs/s", "cores": cores, "kind": "reference",
                         "sample": f"{nb} random base polygons per step joined against all 200000 "
                                   f"overlay polygons (oracle restatement of the join stages), their "
                                   f"clip set clipped by the reference's sequential GH code"},
        "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ----------------------------------------------------------------------------- serving

SERVE_WORKLOAD = ("serving: resident layer of 1,000,000 FP64 stars (batched workload's distributions, "
                  "seed 4) with its MBR grid index in HBM; open-loop Poisson arrivals of query stars "
                  "(vertex counts log-uniform [16, 50000], pool of 512) joined against the layer and "
                  "clipped against every hit")


def _open_loop(srv, queries, rate, seconds, rng, max_requests=None):
    """Submits queries at Poisson arrival times (open loop; latency counts from the
    scheduled arrival, so client lag is charged to the server, never hidden) and returns
    per-request results."""
    n = int(rate * seconds)
    if max_requests:
        n = min(n, max_requests)
    gaps = rng.exponential(1.0 / rate, size=n)
    t0 = time.monotonic_ns() + 2_000_000
    arrivals = t0 + np.cumsum(gaps * 1e9).astype(np.int64)
    pick = rng.integers(0, len(queries), size=n)
    tickets = []
    i = 0
    while i < n:
        now = time.monotonic_ns()
        while i < n and arrivals[i] <= now:
            tickets.append(srv.submit(queries[pick[i]], arrival_ns=int(arrivals[i])))
            i += 1
        if i < n and arrivals[i] > now + 200_000:
            time.sleep(max(0.0, (arrivals[i] - now) * 1e-9 - 1e-4))
    infos = [srv.wait(t, 600_000) for t in tickets]
    for t, inf in zip(tickets, infos):
        srv.take(t, inf)
    return infos, arrivals


def _latency_summary(infos, arrivals, rate):
    lat = np.array([inf["done_ns"] - inf["arrival_ns"] for inf in infos], dtype=np.float64) * 1e-6
    hits = sum(inf["n_hits"] for inf in infos)
    span = (max(inf["done_ns"] for inf in infos) - int(arrivals[0])) * 1e-9
    bad = sum(1 for inf in infos if inf["status"] != 0)
    return {"rate_req_s": rate, "requests": len(infos), "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "pairs_per_s": hits / span,
            "queries_per_s": len(infos) / span, "mean_batch": float(np.mean([inf["batch_queries"] for inf in infos])),
            "errors": bad}


def serve_measure(local, seconds=0.5):
    """p50/p99 latency and pairs/s of the continuous-batching server at 2k/10k/50k req/s,
    and of the plain one-query-per-launch form (one worker, batches of one query)."""
    import gcmfgh
    from gcmfgh import synth
    resident, queries = synth.serving_workload(seed=4)
    rng = np.random.default_rng(44)
    out = {"workload": SERVE_WORKLOAD, "batched": [], "plain": []}
    with gcmfgh.Server(resident, device=local, workers=2) as srv:
        _open_loop(srv, queries, 2000, 0.1, rng)                     # warm-up
        for rate in (2000, 10000, 50000):
            infos, arr = _open_loop(srv, queries, rate, seconds, rng)
            out["batched"].append(_latency_summary(infos, arr, rate))
        out["batched_stats"] = srv.stats()
    with gcmfgh.Server(resident, device=local, workers=1, max_batch_queries=1) as srv:
        _open_loop(srv, queries, 500, 0.1, rng)
        for rate in (2000, 10000, 50000):
            infos, arr = _open_loop(srv, queries, rate, seconds, rng, max_requests=2000)
            out["plain"].append(_latency_summary(infos, arr, rate))
    return out


# ----------------------------------------------------------------------------- plain form

def plain_measure(eng, db, do, stream, n=2000, seed=9):
    """The plain one-pair-per-launch form on the same GPU: a seeded sample of the clip set
    of the last join, each pair clipped by its own gh_clip_batch_host_ids call (its own
    launch sequence, host synchronisations included), same kernels and arithmetic."""
    import ctypes
    import torch
    import gcmfgh
    cb, co = eng.join_field("clip_b"), eng.join_field("clip_o")
    rng = np.random.default_rng(seed)
    idx = rng.choice(len(cb), size=min(n, len(cb)), replace=False)
    L = gcmfgh.lib()
    info = gcmfgh.ClipInfo()
    pids = [np.ascontiguousarray(cb[i:i + 1]) for i in idx]
    qids = [np.ascontiguousarray(co[i:i + 1]) for i in idx]

    def one(k):
        gcmfgh._check(L.gh_clip_batch_host_ids(eng.h, ctypes.byref(db.c), ctypes.byref(do.c),
                                               ctypes.c_void_p(pids[k].ctypes.data),
                                               ctypes.c_void_p(qids[k].ctypes.data), 1, ctypes.byref(info)))
    for k in range(min(50, len(idx))):
        one(k)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(len(idx)):
        one(k)
    e1.record(stream)
    e1.synchronize()
    secs = e0.elapsed_time(e1) * 1e-3
    return {"value": len(idx) / secs, "unit": "pairs/s",
            "sample": f"{len(idx)} seeded pairs of the clip set, one gh_clip_batch call each"}


# ----------------------------------------------------------------------------- precision

def precision_measure(local, n=2000, n_check=150):
    """The degeneracy-stressed batch (independent pairs, vertex counts log-uniform on
    [4, 10000]; 2% share a vertex exactly, 1% have collinear overlapping edges, 1% are
    translated by 1e-12 relative; seed 3), a seeded sample of n pairs: clipped in exact
    mode and in the reference's tolerance mode, timed with CUDA events; the exact results
    of n_check pairs (every degenerate one among them) compared with the oracle."""
    import torch
    import gcmfgh
    import pyoracle
    from gcmfgh import synth
    classes, pairs = synth.degeneracy_pairs(3, n, 4, 10_000)
    base = synth.Layer.from_rings([p for p, _ in pairs])
    ovl = synth.Layer.from_rings([q for _, q in pairs])
    ids = np.arange(n, dtype=np.int32)
    eng = gcmfgh.Engine(local)
    db, do = gcmfgh.DeviceLayer(base, f"cuda:{local}"), gcmfgh.DeviceLayer(ovl, f"cuda:{local}")
    out = {"workload": "degeneracy batch: %d pairs, vertex counts log-uniform [4, 10000], classes "
                       "shared-vertex / collinear-overlap / 1e-12-translated at 2%%/1%%/1%%, seed 3" % n}
    for exact in (True, False):
        eng.set_precision(exact)
        eng.clip_batch(db, do, ids, ids)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        info = eng.clip_batch(db, do, ids, ids)
        e1.record()
        e1.synchronize()
        key = "exact" if exact else "reference_mode"
        out[key] = {"pairs_per_s": n / (e0.elapsed_time(e1) * 1e-3), "invalid_pairs": info["n_invalid"],
                    "errors": info["n_error"]}
        if exact:
            r = eng.clip_result()
    eng.set_precision(False)
    rng = np.random.default_rng(33)
    degenerate = np.flatnonzero(classes > 0)
    rest = np.setdiff1d(np.arange(n), degenerate)
    chk = np.sort(np.concatenate([degenerate, rng.choice(rest, size=max(0, n_check - len(degenerate)), replace=False)]))
    sub_b = synth.Layer.from_rings([pairs[i][0] for i in chk])
    sub_o = synth.Layer.from_rings([pairs[i][1] for i in chk])
    sid = np.arange(len(chk), dtype=np.int32)
    o = pyoracle.clip_batch(sub_b, sub_o, sid, sid, exact=True)
    comps_gpu = [r.components(int(i)) for i in chk]
    comps_orc = [o.components(k) for k in range(len(chk))]
    maxrel = 0.0
    same = True
    for a, b in zip(comps_gpu, comps_orc):
        if len(a) != len(b) or any(x.shape != y.shape for x, y in zip(a, b)):
            same = False
            continue
        for x, y in zip(a, b):
            if x.size:
                maxrel = max(maxrel, float(np.max(np.abs(x - y) / np.maximum(np.abs(y), 1e-300))))
    out["oracle_check"] = {"pairs": int(len(chk)), "degenerate_pairs": int(len(degenerate)),
                           "identical_structure": same, "max_rel_vertex_error": maxrel,
                           "status_equal": bool(np.array_equal(r.status[chk], o.status))}
    eng.close()
    return out


# ----------------------------------------------------------------------------- our arm

def run_ours(args, rank, world, local):
    import torch
    import gcmfgh
    from gcmfgh import synth
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    base, ovl = synth.batched_join(seed=2 + rank)
    eng = gcmfgh.Engine(local)
    stream = torch.cuda.current_stream()
    eng.set_stream(stream.cuda_stream)
    eng.set_timing(True)
    db, do = gcmfgh.DeviceLayer(base, f"cuda:{local}"), gcmfgh.DeviceLayer(ovl, f"cuda:{local}")
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=f"cuda:{local}")

    def step():
        ji = eng.join(db, do)
        ci = eng.clip_joined(db, do)
        return ji, ci

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(local) if rank == 0 else None
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
    l0 = gcmfgh.launch_count()
    times, stages, infos = [], {}, None
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        infos = step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        for which in (0, 1):
            for name, ms in eng.timing(which):
                stages.setdefault(name, []).append(ms)
    torch.cuda.synchronize()
    launches = gcmfgh.launch_count() - l0
    if dist:
        dist.barrier()
    clocks = sampler.stop() if sampler else None
    ji, ci = infos
    ms = statistics.mean(times)
    pairs = ci["n_pairs"]

    # ---- end to end: host (pinned) layers in, result vertices out, every step
    pinned = []
    for L in (base, ovl):
        t = [torch.from_numpy(a).pin_memory() for a in (L.xy, L.vnum, L.vps)]
        pinned.append((t, gcmfgh.Layer(t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), L.n_polys,
                                       L.n_vertices)))
    h2d = sum(int(a.nbytes) for L in (base, ovl) for a in (L.xy, L.vnum, L.vps))
    out_xy = torch.empty(2 * ci["n_vertices"] + 1024, dtype=torch.float64).pin_memory()
    out_cs = torch.empty(ci["n_components"] + 1024, dtype=torch.int32).pin_memory()
    out_nc = torch.empty(pairs + 1024, dtype=torch.int32).pin_memory()
    import ctypes

    def e2e_step():
        jinfo, cinfo = gcmfgh.JoinInfo(), gcmfgh.ClipInfo()
        gcmfgh._check(gcmfgh.lib().gcmfgh_join_clip_host(eng.h, ctypes.byref(pinned[0][1]),
                                                         ctypes.byref(pinned[1][1]), ctypes.byref(jinfo),
                                                         ctypes.byref(cinfo)))
        nbytes = ctypes.c_int64()
        d2h = 0
        for fid, buf in ((6, out_xy), (4, out_cs), (1, out_nc)):
            gcmfgh._check(gcmfgh.lib().gh_clip_get(eng.h, fid, ctypes.c_void_p(buf.data_ptr()),
                                                   buf.numel() * buf.element_size(), 0, ctypes.byref(nbytes)))
            d2h += nbytes.value
        return cinfo.n_pairs, d2h

    for _ in range(max(1, args.warmup // 2)):
        e2e_step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e2e_times, d2h = [], 0
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _, d2h = e2e_step()
        e1.record(stream)
        e1.synchronize()
        e2e_times.append(e0.elapsed_time(e1))
    e2e_ms = statistics.mean(e2e_times)

    # ---- across ranks: slowest rank's time, all ranks' pairs
    if dist:
        t = torch.tensor([ms, e2e_ms], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, e2e_ms = float(t[0]), float(t[1])
        p = torch.tensor([pairs], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(p, op=dist.ReduceOp.SUM)
        total_pairs = float(p[0])
    else:
        total_pairs = float(pairs)

    if rank == 0:
        stage_ms = {k: statistics.mean(v) for k, v in stages.items()}
        dom = max(stage_ms, key=stage_ms.get)
        peak, peak_kind = measured_peaks()
        jb, jo = eng.join_field("b"), eng.join_field("o")
        cand_v = int(base.vnum[jb].astype(np.int64).sum() + ovl.vnum[jo].astype(np.int64).sum())
        counts = (ji, ci, base.n_polys, ovl.n_polys, base.n_vertices, ovl.n_vertices, cand_v)
        alg = stage_bytes(dom, *counts)
        achieved = (alg / (stage_ms[dom] * 1e-3) / 1e9) if alg else None
        # every stage with a byte model, and the whole step: sum of algorithmic bytes / step time
        per_stage = {}
        for k, v in stage_ms.items():
            b = stage_bytes(k, *counts)
            if b:
                per_stage[k] = {"ms": round(v, 4), "algorithmic_bytes": b,
                                "frac": round(b / (v * 1e-3) / 1e9 / peak, 5)}
        step_bytes = (32 * (base.n_polys + ovl.n_polys) + 8 * ji["n_pairs"] + 16 * cand_v
                      + 16 * ci["n_ring_vertices"] + 16 * ci["n_vertices"] + 8 * pairs)
        line = {
            "metric": METRIC, "value": total_pairs / (ms * 1e-3), "unit": "pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "pairs_per_step_per_gpu": pairs,
                       "candidates_per_step_per_gpu": ji["n_pairs"], "parallelism": f"replicas{world}",
                       "l2": "flushed between steps (256 MiB write, outside the step events)",
                       "inputs_resident": True},
            "e2e": {"value": total_pairs / (e2e_ms * 1e-3), "unit": "pairs/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": traffic_from_profiles(dom),
                         "algorithmic_bytes": alg, "kernel_ms": stage_ms[dom], "peak_source": peak_kind},
            "stages_ms": {k: round(v, 4) for k, v in stage_ms.items()},
            "stage_roofline": per_stage,
            "step_roofline": {"algorithmic_bytes": step_bytes, "achieved": step_bytes / (ms * 1e-3) / 1e9,
                              "peak": peak, "unit": "GB/s", "frac": step_bytes / (ms * 1e-3) / 1e9 / peak,
                              "bytes": "32 B per layer MBR + 8 B per candidate pair + 16 B per vertex of "
                                       "both polygons of every candidate (CMF edge scan) + 16 B per merged "
                                       "ring vertex + 16 B per result vertex + 8 B per clipped pair"},
            "clocks": clocks,
            "gpu_launches": launches,
        }
        plain = plain_measure(eng, db, do, stream)
        plain["batched_over_plain"] = line["value"] / world / plain["value"]
        line["plain"] = plain
        if not args.no_serve:
            line["serving"] = serve_measure(local)
            line["precision"] = precision_measure(local)
        if world == 1 and not args.no_cpu_baseline:
            nb = args.sample_bases or 20000
            p, s, cores = reference_cpu_sample(base, ovl, nb, 7)
            line["cpu_baseline"] = {"value": p / s, "unit": "pairs/s", "cores": cores, "kind": "reference",
                                    "sample": f"{nb} random base polygons joined against all overlay "
                                              f"polygons (oracle restatement of the join stages), their "
                                              f"{p} clip pairs clipped by the reference's sequential GH "
                                              f"code built from its sources"}
        print(json.dumps(line), flush=True)
    eng.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
