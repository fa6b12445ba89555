#!/usr/bin/env python
"""Join+clip polygon pairs/s on the batched spatial-join workload.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Workload (one step): the GCMF join of two layers of 200,000 FP64 star polygons (vertex
counts floor(Pareto(1.5, 4)) capped at 100,000; centres from a 64-component Gaussian
mixture over [0,1e5]^2, sigma 2,000; base radius log-normal(ln 50, 0.7); seed 2),
followed by the Greiner-Hormann clip of every pair in the clip set.
The unit is one clipped polygon pair.  Under torchrun the ranks split that one workload:
rank r joins and clips its x-slab of base polygons (equal counts by MBR x1) against the
whole overlay layer, with no data-path collective (strong scaling).

value: each rank runs the K timed steps on --lanes contexts (default 4), each on its own
CUDA stream and host thread and taking every lanes-th step, so that one context's kernels
run while another waits on a size read-back; every step starts with an L2 flush.  The
time is the device time from a common start event to the last lane's end event, the
slowest rank's; value = all ranks' pairs per step x K / that time.  e2e is the same
through gcmfgh_join_clip_host (pinned host layers in, every result array out, each step).
single_lane holds the one-context numbers, whose per-step events give the stage times.

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
    ap.add_argument("--precision-pairs", type=int, default=1_000_000, help="pairs of the degeneracy batch")
    ap.add_argument("--precision-chunk", type=int, default=50_000, help="pairs generated and clipped at once")
    ap.add_argument("--precision-check-all", action="store_true",
                    help="compare every degenerate pair (not a sample) with the oracle")
    ap.add_argument("--no-precision", action="store_true", help="skip the degeneracy batch")
    ap.add_argument("--no-large-pair", action="store_true", help="skip the single large pair")
    ap.add_argument("--no-multi", action="store_true", help="skip the multi-component pairs")
    ap.add_argument("--join-sweep", type=int, default=None,
                    help="1: MBR candidates by the sort-sweep, 0: by the grid probe (default: the library's)")
    ap.add_argument("--lanes", type=int, default=4,
                    help="contexts (and host threads) of the pipelined measurement; 1 skips it")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default size-bucket thresholds")
    ap.add_argument("--fused-emit", type=int, default=None,
                    help="0: count, then emit the intersection records; 1: one pass, block-wide "
                         "appends; 2: one pass, warp appends (default: the library's)")
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
        "clip:count+emit": 16 * ring + 8 * C + 33 * recs,
        "join:mbr+sort": 16 * (vb + vo) + 40 * (nb + no),
        # MBRs of both layers, the overlay's extent and its grid listing
        "join:mbr+grid": 16 * (vb + vo) + 36 * (nb + no) + 4 * no,
        # each base MBR probes its cells; each listed overlay MBR it meets is read
        "join:cand-count": 32 * (nb + no),
        "join:cand-emit+sort": 32 * (nb + no) + 16 * K,
        "join:sweep-count": 36 * (nb + no),
        "join:sweep-emit+sort": 36 * (nb + no) + 16 * K,
        # one-pass sweep: the x1-sorted MBRs read once, the keys written; then their sort
        "join:sweep": 36 * (nb + no) + 8 * K,
        "join:sort": 16 * K,
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


def serve_measure(local, seconds=2.0):
    """p50/p99 latency and pairs/s of the continuous-batching server at 2k/10k/50k req/s,
    and of the plain one-query-per-launch form (one worker, batches of one query)."""
    import gcmfgh
    from gcmfgh import synth
    resident, queries = synth.serving_workload(seed=4)
    rng = np.random.default_rng(44)
    out = {"workload": SERVE_WORKLOAD, "batched": [], "plain": []}
    with gcmfgh.Server(resident, device=local, workers=4) as srv:
        _open_loop(srv, queries, 2000, 0.1, rng)                     # warm-up
        for rate in (2000, 10000, 50000):
            ms0, w0 = srv.phases()
            infos, arr = _open_loop(srv, queries, rate, seconds, rng)
            ms1, w1 = srv.phases()
            summ = _latency_summary(infos, arr, rate)
            tot = sum(ms1[k] - ms0[k] for k in ms1) or 1.0
            summ["phase_share"] = {k: round((ms1[k] - ms0[k]) / tot, 4) for k in ms1}
            summ["phase_ms_summed"] = {k: round(ms1[k] - ms0[k], 2) for k in ms1}
            summ["work"] = {k: w1[k] - w0[k] for k in w1}
            out["batched"].append(summ)
        out["batched_stats"] = srv.stats()
    with gcmfgh.Server(resident, device=local, workers=1, max_batch_queries=1) as srv:
        _open_loop(srv, queries, 500, 0.1, rng)
        for rate in (2000, 10000, 50000):
            infos, arr = _open_loop(srv, queries, rate, seconds, rng, max_requests=1000)
            out["plain"].append(_latency_summary(infos, arr, rate))
    return out


# ----------------------------------------------------------------------------- plain form

def plain_measure(eng, db, do, stream, n=2000, seed=9):
    """The plain one-pair-per-launch form on the same GPU and the same resident context: a
    seeded sample of the clip set of the last join, each pair run through the whole join +
    clip pipeline on its own (gcmf_join over one-polygon views of the two device layers,
    then gh_clip_joined: every launch sequence and host synchronisation of the batched
    step, for one pair), same kernels and arithmetic.  Pairs/s of that form is the
    denominator of batched_over_plain."""
    import ctypes
    import torch
    import gcmfgh
    cb, co = eng.join_field("clip_b"), eng.join_field("clip_o")
    rng = np.random.default_rng(seed)
    idx = rng.choice(len(cb), size=min(n, len(cb)), replace=False)
    L = gcmfgh.lib()
    dev = db.xy.device
    views = []
    for lay, ids in ((db, cb[idx]), (do, co[idx])):
        vnum = lay.layer.vnum[ids].astype(np.int32)
        start = (lay.layer.vps[ids] - lay.layer.vnum[ids]).astype(np.int64)
        dv = torch.from_numpy(vnum).to(dev)             # one polygon per view: vps = vnum
        dp = torch.from_numpy(vnum.astype(np.int64)).to(dev)
        views.append((dv, dp, start, vnum))
    (bv, bp, bs, bn), (ov, op, os_, on) = views
    esz = db.xy.element_size()
    lb = [gcmfgh.Layer(db.xy.data_ptr() + 2 * esz * int(bs[k]), bv.data_ptr() + 4 * k, bp.data_ptr() + 8 * k, 1,
                       int(bn[k])) for k in range(len(idx))]
    lo = [gcmfgh.Layer(do.xy.data_ptr() + 2 * esz * int(os_[k]), ov.data_ptr() + 4 * k, op.data_ptr() + 8 * k, 1,
                       int(on[k])) for k in range(len(idx))]
    ji, ci = gcmfgh.JoinInfo(), gcmfgh.ClipInfo()
    clipped = 0

    def one(k):
        gcmfgh._check(L.gcmf_join(eng.h, ctypes.byref(lb[k]), ctypes.byref(lo[k]), ctypes.byref(ji)))
        gcmfgh._check(L.gh_clip_joined(eng.h, ctypes.byref(lb[k]), ctypes.byref(lo[k]), ctypes.byref(ci)))
        return ci.n_pairs

    for k in range(min(50, len(idx))):
        one(k)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(len(idx)):
        clipped += one(k)
    e1.record(stream)
    e1.synchronize()
    secs = e0.elapsed_time(e1) * 1e-3
    # restore the batched join's state for the caller
    eng.join(db, do)
    return {"value": clipped / secs, "unit": "pairs/s", "pairs_clipped": int(clipped),
            "sample": f"{len(idx)} seeded pairs of the clip set, each run alone through gcmf_join + "
                      f"gh_clip_joined on one-polygon views of the resident layers"}


# ----------------------------------------------------------------------------- single large pair

def pipelined_measure(local, db, do, pinned, out_sizes, tuning, steps, warmup, lanes, fused_emit,
                      join_sweep=None):
    """Whole-job throughput of `lanes` contexts on one GPU, each on its own stream, driven by
    its own host thread and taking every lanes-th step, all with the same thresholds: while
    one context waits on a size read-back or on PCIe, the others' kernels run.  Each step
    starts with an L2 flush (a 256 MiB write on the lane's stream, inside the timed region).
    Timed on the device: an event on the main stream that every lane's stream waits on
    before its first step, to the last of the lanes' end events.  Two forms:
    resident (gcmf_join + gh_clip_joined on the device layers) and end to end
    (gcmfgh_join_clip_host from the pinned host layers, every result array read back into
    pinned host buffers).  Returns ms per step of both, launches per step, and the result
    bytes read back per step."""
    import ctypes
    import threading
    import torch
    import gcmfgh
    engines = [gcmfgh.Engine(local) for _ in range(lanes)]
    streams = [torch.cuda.Stream(device=f"cuda:{local}") for _ in range(lanes)]
    flush = [torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=f"cuda:{local}") for _ in range(lanes)]
    for e, st in zip(engines, streams):
        e.set_stream(st.cuda_stream)
        e.set_tuning(**tuning)
        if fused_emit is not None:
            e.set_tuning(fused_emit=fused_emit)
        if join_sweep is not None:
            e.set_tuning(join_sweep=bool(join_sweep))
    outs = [(torch.empty(out_sizes[0], dtype=torch.float64).pin_memory(),
             torch.empty(out_sizes[1], dtype=torch.int32).pin_memory(),
             torch.empty(out_sizes[2], dtype=torch.int32).pin_memory()) for _ in range(lanes)]
    L = gcmfgh.lib()
    d2h = [0] * lanes

    def resident(j):
        engines[j].join(db, do)
        engines[j].clip_joined(db, do)

    def e2e(j):
        eng = engines[j]
        jinfo, cinfo = gcmfgh.JoinInfo(), gcmfgh.ClipInfo()
        gcmfgh._check(L.gcmfgh_join_clip_host(eng.h, ctypes.byref(pinned[0][1]), ctypes.byref(pinned[1][1]),
                                              ctypes.byref(jinfo), ctypes.byref(cinfo)))
        nbytes = ctypes.c_int64()
        total = 0
        for fid, buf in zip((6, 4, 1), outs[j]):
            gcmfgh._check(L.gh_clip_get(eng.h, fid, ctypes.c_void_p(buf.data_ptr()), buf.numel() * buf.element_size(),
                                        0, ctypes.byref(nbytes)))
            total += nbytes.value
        d2h[j] = total

    def run(fn, n):
        errs = []
        gate = threading.Barrier(lanes + 1)
        start = torch.cuda.Event(enable_timing=True)
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(lanes)]

        def worker(j):
            try:
                gate.wait()
                streams[j].wait_event(start)
                for _ in range(j, n, lanes):
                    with torch.cuda.stream(streams[j]):
                        flush[j].zero_()
                    fn(j)
                ends[j].record(streams[j])
            except Exception as e:          # reported after the join
                errs.append(e)
        th = [threading.Thread(target=worker, args=(j,)) for j in range(lanes)]
        for t in th:
            t.start()
        torch.cuda.synchronize()
        l0 = gcmfgh.launch_count()
        start.record(torch.cuda.current_stream())
        gate.wait()
        for t in th:
            t.join()
        torch.cuda.synchronize()
        if errs:
            raise errs[0]
        ms = max(start.elapsed_time(e) for e in ends[:min(lanes, n)])
        return ms / n, (gcmfgh.launch_count() - l0) / n

    try:
        run(resident, max(warmup, lanes))
        res_ms, res_launches = run(resident, steps)
        run(e2e, max(warmup, lanes))
        e2e_ms, _ = run(e2e, steps)
    finally:
        for e in engines:
            e.close()
    return {"lanes": lanes, "resident_ms_per_step": res_ms, "e2e_ms_per_step": e2e_ms,
            "launches_per_step": res_launches, "d2h_bytes_per_step": d2h[0]}


def multi_measure(local, n=5000, single=300, seed=41):
    """Multi-component pairs (islands with 0-3 holes, 5-200 vertices per ring, seeded):
    n pairs through one gh_clip_multi_batch call, against `single` of them through one
    gh_clip_multi call each.  Host arrays in, results on the device; wall clock around
    synchronised calls."""
    import torch
    import gcmfgh
    from gcmfgh import synth
    pairs = synth.holed_pairs(seed, n, 5, 200)
    eng = gcmfgh.Engine(local)
    try:
        eng.clip_multi_batch(pairs[:100])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        info = eng.clip_multi_batch(pairs)
        torch.cuda.synchronize()
        tb = time.perf_counter() - t0
        for P, Q in pairs[:10]:
            eng.clip_multi(P, Q)
        t0 = time.perf_counter()
        for P, Q in pairs[:single]:
            eng.clip_multi(P, Q)
        torch.cuda.synchronize()
        ts = time.perf_counter() - t0
    finally:
        eng.close()
    rings = sum(len(P) + len(Q) for P, Q in pairs)
    return {"workload": f"{n} seeded pairs of islands with holes (holed_pairs seed {seed}, 5-200 vertices "
                        f"per ring, {rings} rings), P and Q as given",
            "batch_pairs_per_s": n / tb, "batch_ms": tb * 1e3, "records": info["n_records"],
            "components_out": info["n_components"],
            "single_call_pairs_per_s": single / ts, "batch_over_single": (n / tb) / (single / ts)}


def large_pair_measure(local, nP=1_000_000, nQ=500_000, reps=2, cpu_div=64):
    """The single large pair (star of nP vertices, radius U(0.8,1.2), at the origin, clipped
    by a star of nQ vertices, radius U(0.7,1.3), centred at (0.05, 0.03); seed 1) in exact
    mode, timed with CUDA events after one warm-up clip.  The reference's sequential
    clipper tests every edge pair (O(nP nQ), 5e11 tests here) and inserts each intersection
    into linked lists, so its time is taken on the same distribution at nP/cpu_div x
    nQ/cpu_div vertices and scaled by cpu_div^2 -- an extrapolation and a lower bound, as
    the sample times grow faster than quadratically."""
    import torch
    import gcmfgh
    import pyoracle
    from gcmfgh import synth
    s, c = synth.large_pair(1, nP, nQ)
    eng = gcmfgh.Engine(local)
    eng.set_timing(True)
    ds, dc = gcmfgh.DeviceLayer(s, f"cuda:{local}"), gcmfgh.DeviceLayer(c, f"cuda:{local}")
    one = np.array([0], np.int32)
    eng.set_precision(True)
    info = eng.clip_batch(ds, dc, one, one)
    times = []
    for _ in range(reps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        info = eng.clip_batch(ds, dc, one, one)
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    stages = {k: round(v, 2) for k, v in eng.timing(1)}
    st = eng.clip_field("status")
    eng.set_precision(False)
    eng.close()
    out = {"workload": f"single large pair: {nP} x {nQ} vertex stars (seed 1), exact mode",
           "gpu_s": min(times) * 1e-3, "status": int(st[0]), "intersection_records": info["n_records"],
           "components": info["n_components"], "vertices": info["n_vertices"], "stages_ms": stages}
    if pyoracle.ref_available():
        sp, cp = synth.large_pair(1, nP // cpu_div, nQ // cpu_div)
        P, Q = sp.ring(0), cp.ring(0)
        with tempfile.TemporaryDirectory() as td:
            fn = os.path.join(td, "lp.bin")
            pyoracle.write_pair_batch(fn, [(P, Q)])
            r = subprocess.run([pyoracle.REF_BIN, "time", fn, "1"], stdout=subprocess.PIPE, text=True, check=True)
            t = float(r.stdout.split()[0])
        out["cpu_reference"] = {"sample_s": t, "sample": f"{len(P)} x {len(Q)} vertices, one core",
                                "extrapolated_s": t * cpu_div * cpu_div,
                                "method": f"lower bound: sample time x {cpu_div}^2 for the O(nP nQ) edge "
                                          f"tests (the sample times grow faster than that: 0.85 s at "
                                          f"half these sizes)"}
        out["gpu_over_cpu_extrapolated"] = out["cpu_reference"]["extrapolated_s"] / out["gpu_s"]
    return out


# ----------------------------------------------------------------------------- precision

def _area(comps):
    """Total signed shoelace area of a result's components."""
    a = 0.0
    for c in comps:
        if len(c) >= 3:
            x, y = c[:, 0], c[:, 1]
            a += 0.5 * float(np.dot(x, np.roll(y, -1)) - np.dot(np.roll(x, -1), y))
    return a


def _compare(gpu_st, gpu_comps, orc):
    """Parity of GPU results against the oracle's: status and component structure equal,
    max relative vertex error, max relative area error."""
    same_status = bool(np.array_equal(gpu_st, orc.status))
    same_structure = True
    max_v = max_a = 0.0
    for k, a in enumerate(gpu_comps):
        b = orc.components(k)
        if len(a) != len(b) or any(x.shape != y.shape for x, y in zip(a, b)):
            same_structure = False
            continue
        for x, y in zip(a, b):
            if x.size:
                max_v = max(max_v, float(np.max(np.abs(x - y) / np.maximum(np.abs(y), 1e-300))))
        aa, ab = _area(a), _area(b)
        if aa != ab:
            max_a = max(max_a, abs(aa - ab) / max(abs(ab), 1e-300))
    return {"status_equal": same_status, "identical_structure": same_structure,
            "max_rel_vertex_error": max_v, "max_rel_area_error": max_a}


def precision_measure(local, total=1_000_000, chunk=50_000, check_degenerate=1200, check_generic=600,
                      check_all_degenerate=False):
    """The degeneracy-stressed batch at its full size: `total` independent pairs (vertex
    counts log-uniform on [4, 10000]; 2% share a vertex exactly, 1% have collinear
    overlapping edges, 1% are translated by 1e-12 relative; seed 3), generated on the GPU
    in chunks of `chunk` pairs and clipped chunk by chunk in exact mode and in the
    reference's tolerance mode (eps 1e-7), each clip timed with CUDA events.  A stratified
    sample -- `check_degenerate` degenerate and `check_generic` generic pairs spread over
    the chunks (every degenerate pair with check_all_degenerate) -- is compared with the
    FP64 oracle in both modes: status, component structure, relative vertex and area
    error.  Pairs that end in status 3 are the ones whose trace does not close: the
    reference's own clipper loops on them (its trace appends vertices without end), the
    engine and the oracle stop the walk and report the pair."""
    import torch
    import gcmfgh
    import pyoracle
    from gcmfgh import synth
    dev = torch.device("cuda", local)
    eng = gcmfgh.Engine(local)
    nchunks = (total + chunk - 1) // chunk
    modes = {"exact": True, "reference_mode": False}
    agg = {m: {"pairs": 0, "ms": 0.0, "invalid_pairs": 0, "errors": 0, "disjoint_pairs": 0, "components": 0,
               "vertices": 0, "records": 0} for m in modes}
    classes_all = np.zeros(4, np.int64)
    rng = np.random.default_rng(33)
    samples = {m: [] for m in modes}          # (P ring, Q ring, status, components)
    per_deg = (check_degenerate + nchunks - 1) // nchunks
    per_gen = (check_generic + nchunks - 1) // nchunks
    for c in range(nchunks):
        n = min(chunk, total - c * chunk)
        cls, B, O = synth.degeneracy_chunk_device(3, c, n, device=dev)
        classes_all += np.bincount(cls, minlength=4)
        db, do = gcmfgh.DeviceLayer.from_tensors(*B), gcmfgh.DeviceLayer.from_tensors(*O)
        ids = torch.arange(n, dtype=torch.int32, device=dev)
        deg = np.flatnonzero(cls > 0)
        gen = np.flatnonzero(cls == 0)
        if not check_all_degenerate:
            deg = rng.choice(deg, size=min(per_deg, len(deg)), replace=False)
        sel = np.sort(np.concatenate([deg, rng.choice(gen, size=min(per_gen, len(gen)), replace=False)]))
        bv, bp = B[1].cpu().numpy(), B[2].cpu().numpy()
        ov, op = O[1].cpu().numpy(), O[2].cpu().numpy()
        rings = []
        for k in sel:
            k = int(k)
            pb = B[0][2 * (bp[k] - bv[k]):2 * (bp[k] - 1)].cpu().numpy().reshape(-1, 2)
            pq = O[0][2 * (op[k] - ov[k]):2 * (op[k] - 1)].cpu().numpy().reshape(-1, 2)
            rings.append((pb, pq, int(cls[k])))
        for m, exact in modes.items():
            eng.set_precision(exact)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            info = eng.clip_batch(db, do, ids, ids)
            e1.record()
            e1.synchronize()
            a = agg[m]
            a["pairs"] += n
            a["ms"] += e0.elapsed_time(e1)
            a["invalid_pairs"] += info["n_invalid"]
            a["errors"] += info["n_error"]
            a["disjoint_pairs"] += info["n_disjoint"]
            a["components"] += info["n_components"]
            a["vertices"] += info["n_vertices"]
            a["records"] += info["n_records"]
            if info["n_error"]:
                stat = eng.clip_field("status")
                a.setdefault("errors_by_class", np.zeros(4, np.int64))
                a["errors_by_class"] += np.bincount(cls[stat == 3], minlength=4)
            st, comps = eng.clip_result_pairs(sel)
            samples[m].extend((r[0], r[1], s_, cc, r[2]) for r, s_, cc in zip(rings, st, comps))
        del db, do, B, O
    eng.set_precision(False)
    eng.close()
    out = {"workload": "degeneracy batch: %d pairs generated on the GPU in chunks of %d, vertex counts "
                       "log-uniform [4, 10000], classes shared-vertex / collinear-overlap / "
                       "1e-12-translated at 2%%/1%%/1%%, seed 3" % (total, chunk),
           "pairs": total, "classes": {"generic": int(classes_all[0]), "shared_vertex": int(classes_all[1]),
                                       "collinear_overlap": int(classes_all[2]),
                                       "translated_1e-12": int(classes_all[3])}}
    for m, exact in modes.items():
        a = agg[m]
        sub_b = synth.Layer.from_rings([r[0] for r in samples[m]])
        sub_o = synth.Layer.from_rings([r[1] for r in samples[m]])
        sid = np.arange(len(samples[m]), dtype=np.int32)
        t0 = time.perf_counter()
        o = pyoracle.clip_batch(sub_b, sub_o, sid, sid, exact=exact)
        t_orc = time.perf_counter() - t0
        chk = _compare(np.array([s_[2] for s_ in samples[m]]), [s_[3] for s_ in samples[m]], o)
        chk.update({"pairs": len(sid), "degenerate_pairs": int(sum(1 for x in samples[m] if x[4] > 0)),
                    "oracle_s": round(t_orc, 2), "status3_pairs_in_sample": int(np.sum(o.status == 3))})
        out[m] = {"pairs_per_s": a["pairs"] / (a["ms"] * 1e-3), "ms_total": a["ms"],
                  "invalid_pairs": a["invalid_pairs"], "errors": a["errors"], "disjoint_pairs": a["disjoint_pairs"],
                  "components": a["components"], "vertices": a["vertices"], "records": a["records"],
                  "errors_by_class": dict(zip(("generic", "shared_vertex", "collinear_overlap", "translated_1e-12"),
                                              [int(x) for x in a.get("errors_by_class", np.zeros(4))])),
                  "oracle_check": chk}
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
    from gcmfgh import shard
    full_base, ovl = synth.batched_join(seed=2)
    # one workload split across the ranks: rank r joins and clips its x-slab of base
    # polygons against the whole overlay layer (every pair is found by exactly one rank)
    base, _ = shard.shard_base(full_base, world, rank) if world > 1 else (full_base, None)
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

    if args.fused_emit is not None:
        eng.set_tuning(fused_emit=args.fused_emit)
    if args.join_sweep is not None:
        eng.set_tuning(join_sweep=bool(args.join_sweep))
    # the autotuner picks the size-bucket thresholds for this workload (outside the timing)
    eng.join(db, do)
    if args.no_autotune:
        ci0 = eng.clip_joined(db, do)
        tuning = eng.tuning_for(db, do, ci0["n_pairs"])
    else:
        tuning = eng.autotune_joined(db, do)

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

    # ---- the same two measurements with two contexts, each driven by its own host thread
    # and taking every other step: one context's kernels run while the other waits on a
    # size read-back or on PCIe
    pipe = None
    if args.lanes > 1:
        pipe = pipelined_measure(local, db, do, pinned, (out_xy.numel(), out_cs.numel(), out_nc.numel()),
                                 {k: tuning[k] for k in ("bin_grid", "tile_label", "mid_label", "big_label",
                                                         "wide_label")},
                                 args.steps, args.warmup, args.lanes, args.fused_emit, args.join_sweep)

    # the clocks were sampled through the single-lane, end-to-end and pipelined regions
    clocks = sampler.stop() if sampler else None
    # the headline numbers: the pipelined form when it ran, else the single-lane one
    v_ms = pipe["resident_ms_per_step"] if pipe else ms
    v_e2e_ms = pipe["e2e_ms_per_step"] if pipe else e2e_ms
    v_launches = int(round(pipe["launches_per_step"] * args.steps)) if pipe else launches

    # ---- across ranks: slowest rank's time, all ranks' pairs
    if dist:
        t = torch.tensor([ms, e2e_ms, v_ms, v_e2e_ms], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, e2e_ms, v_ms, v_e2e_ms = float(t[0]), float(t[1]), float(t[2]), float(t[3])
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
                                "frac": round(b / (v * 1e-3) / 1e9 / peak, 5),
                                "traffic": traffic_from_profiles(k)}
        step_bytes = (32 * (base.n_polys + ovl.n_polys) + 8 * ji["n_pairs"] + 16 * cand_v
                      + 16 * ci["n_ring_vertices"] + 16 * ci["n_vertices"] + 8 * pairs)
        line = {
            "metric": METRIC, "value": total_pairs / (v_ms * 1e-3), "unit": "pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": v_ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "pairs_per_step_rank0": pairs, "pairs_per_step": int(total_pairs),
                       "candidates_per_step_rank0": ji["n_pairs"],
                       "parallelism": f"x-slabs of the base layer over {world} GPU(s), overlay layer replicated",
                       "lanes": pipe["lanes"] if pipe else 1,
                       "l2": ("flushed before every step (256 MiB write on the step's stream, inside the timed "
                              "region)" if pipe else "flushed between steps (256 MiB write, outside the step "
                              "events)"),
                       "inputs_resident": True},
            "e2e": {"value": total_pairs / (v_e2e_ms * 1e-3), "unit": "pairs/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "single_lane": {"value": total_pairs / (ms * 1e-3), "ms_per_step": ms,
                            "e2e": total_pairs / (e2e_ms * 1e-3), "gpu_launches": launches,
                            "note": "one context, one host thread, each step timed alone by CUDA events, L2 "
                                    "flushed between steps outside the events; stages_ms and the rooflines "
                                    "come from these steps"},
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
            "gpu_launches": v_launches,
            "autotune": {"chosen": {k: tuning[k] for k in ("bin_grid", "tile_label", "mid_label", "big_label",
                                                            "wide_label")},
                         "clip_ms_default": tuning["ms_default"], "clip_ms_tuned": tuning["ms_tuned"],
                         "gain": tuning["ms_default"] / tuning["ms_tuned"] if tuning["ms_tuned"] else None,
                         "configs_timed": tuning["configs_timed"]},
        }
        if pipe:
            line["pipelined"] = pipe
        plain = plain_measure(eng, db, do, stream)
        plain["batched_over_plain"] = line["value"] / world / plain["value"]
        line["plain"] = plain
    # the sections below run engines of their own: give back this one's device memory first
    eng.close()
    del db, do, flush, pinned
    torch.cuda.empty_cache()
    if rank == 0:
        # the one-GPU sections (serving, single large pair, multi-component pairs, degeneracy
        # batch) run at N = 1 only: under torchrun the other ranks' GPUs would wait idle
        if not args.no_serve and world == 1:
            line["serving"] = serve_measure(local)
        if not args.no_large_pair and world == 1:
            line["large_pair"] = large_pair_measure(local)
        if not args.no_multi and world == 1:
            line["multi_component"] = multi_measure(local)
        if not args.no_precision and world == 1:
            line["precision"] = precision_measure(local, total=args.precision_pairs, chunk=args.precision_chunk,
                                                  check_all_degenerate=args.precision_check_all)
        if world == 1 and not args.no_cpu_baseline:
            nb = args.sample_bases or 20000
            p, s, cores = reference_cpu_sample(base, ovl, nb, 7)
            line["cpu_baseline"] = {"value": p / s, "unit": "pairs/s", "cores": cores, "kind": "reference",
                                    "sample": f"{nb} random base polygons joined against all overlay "
                                              f"polygons (oracle restatement of the join stages), their "
                                              f"{p} clip pairs clipped by the reference's sequential GH "
                                              f"code built from its sources"}
        print(json.dumps(line), flush=True)
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
