"""The single-large-pair workload in exact-predicate mode, checked bit-exactly at every
size in tests/golden/large_pair_digests.json (the oracle's own results, digested by
tests/golden/make_large_pair_digests.py), up to the full 1,000,000 x 500,000 vertices:
status, intersection count, component count, vertex count and SHA-256 of the component
sizes and of every output coordinate."""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from gcmfgh import synth

pytestmark = pytest.mark.gpu

DIGESTS = os.path.join(GOLDEN, "large_pair_digests.json")
SIZES = sorted(json.load(open(DIGESTS)).items(), key=lambda kv: kv[1]["count1"]) if os.path.exists(DIGESTS) else []


@pytest.mark.parametrize("size,want", SIZES, ids=[k for k, _ in SIZES])
def test_large_pair_exact_digest(engine, size, want):
    import gcmfgh
    nP, nQ = (int(v) for v in size.split("x"))
    s, c = synth.large_pair(1, nP, nQ)
    one = np.array([0], np.int32)
    ds, dc = gcmfgh.DeviceLayer(s), gcmfgh.DeviceLayer(c)
    engine.set_precision(True)
    try:
        info = engine.clip_batch(ds, dc, one, one)
        r = engine.clip_result()
    finally:
        engine.set_precision(False)
    assert info["n_error"] == 0
    got = {
        "status": int(r.status[0]), "count1": int(r.count1[0]), "ncomp": int(r.ncomp[0]),
        "nv": int(len(r.xy) // 2),
        "comp_size_sha256": hashlib.sha256(np.ascontiguousarray(r.comp_size, "<i4").tobytes()).hexdigest(),
        "xy_sha256": hashlib.sha256(np.ascontiguousarray(r.xy, "<f8").tobytes()).hexdigest(),
    }
    assert got == {k: want[k] for k in got}
