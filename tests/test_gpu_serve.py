"""Continuous-batching server: every query's hits and clipped components equal the
oracle's join + clip of that query against the resident layer, whether the query is
served alone, in a burst with many others (batched, batches overlapping on the device),
or in the plain one-query-per-launch form."""
import time

import numpy as np
import pytest

import pyoracle
from gcmfgh import synth

pytestmark = pytest.mark.gpu


def _workload(nq=300, exact=False):
    resident, queries = synth.small_join(0, 2000)
    qrings = [queries.ring(i) for i in range(nq)]
    qlayer = synth.Layer.from_rings(qrings)
    j = pyoracle.join(qlayer, resident)
    sel = j.clip == 1
    b, o = j.b[sel], j.o[sel]
    c = pyoracle.clip_batch(qlayer, resident, b, o, exact=exact)
    expect = []
    comp = 0
    vert = 0
    for q in range(nq):
        idx = np.flatnonzero(b == q)
        sizes, xy = [], []
        for k in idx:
            for _ in range(c.ncomp[k]):
                sz = c.comp_size[comp]
                sizes.append(sz)
                xy.append(c.xy[2 * vert:2 * (vert + sz)])
                vert += sz
                comp += 1
        expect.append((o[idx], c.status[idx], c.ncomp[idx], np.array(sizes, np.int32),
                       np.concatenate(xy) if xy else np.zeros(0)))
    assert comp == len(c.comp_size)
    return resident, qrings, expect


def _same(res, exp):
    ids, st, nc, sizes, xy = exp
    return (np.array_equal(res.hit_ids, ids) and np.array_equal(res.hit_status, st)
            and np.array_equal(res.hit_ncomp, nc) and np.array_equal(res.comp_size, sizes)
            and np.array_equal(res.xy, xy))


@pytest.fixture(scope="module")
def workload():
    return _workload()


def test_serve_alone_equals_oracle(workload):
    import gcmfgh
    resident, qrings, expect = workload
    with gcmfgh.Server(resident) as srv:
        for q in range(0, len(qrings), 7):
            r = srv.result(srv.submit(qrings[q]), timeout_ms=60000)
            assert r.info["status"] == 0 and r.info["batch_queries"] == 1
            assert _same(r, expect[q]), q


def test_serve_burst_equals_oracle_and_batches(workload):
    import gcmfgh
    resident, qrings, expect = workload
    with gcmfgh.Server(resident, workers=2) as srv:
        t0 = time.monotonic_ns()
        tickets = [srv.submit(r, arrival_ns=t0) for r in qrings]
        results = [srv.result(t, timeout_ms=120000) for t in tickets]
        stats = srv.stats()
    assert stats["queries"] == len(qrings) and stats["peak_batch"] > 1
    for q, r in enumerate(results):
        assert r.info["status"] == 0
        assert _same(r, expect[q]), q
    # batches were formed from what was waiting: at most as many batches as queries
    assert len({r.info["batch_id"] for r in results}) < len(qrings)


def test_serve_plain_form_equals_oracle(workload):
    import gcmfgh
    resident, qrings, expect = workload
    with gcmfgh.Server(resident, workers=1, max_batch_queries=1) as srv:
        tickets = [srv.submit(r) for r in qrings[:60]]
        for q, t in enumerate(tickets):
            r = srv.result(t, timeout_ms=60000)
            assert r.info["batch_queries"] == 1 and _same(r, expect[q])


def test_serve_exact_mode_and_small_budgets():
    """Exact predicates through the server, with tiny vertex budgets forcing many batches."""
    import gcmfgh
    resident, qrings, expect = _workload(120, exact=True)
    with gcmfgh.Server(resident, workers=3, max_batch_vertices=400, exact=True) as srv:
        tickets = [srv.submit(r) for r in qrings]
        for q, t in enumerate(tickets):
            r = srv.result(t, timeout_ms=60000)
            assert r.info["status"] == 0 and _same(r, expect[q])


def test_serve_rejects_bad_queries(workload):
    import gcmfgh
    resident, _, _ = workload
    with gcmfgh.Server(resident) as srv:
        with pytest.raises(gcmfgh.GcmfghError):
            srv.submit(np.zeros((0, 2)))
