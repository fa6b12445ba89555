"""Several contexts on one GPU, each driven by its own host thread (the pipelined form of
the bench): every context's join + clip results equal a lone context's bit for bit."""
import threading

import numpy as np
import pytest

from gcmfgh import synth

pytestmark = pytest.mark.gpu


def _result(eng, db, do):
    ji = eng.join(db, do)
    ci = eng.clip_joined(db, do)
    r = eng.clip_result()
    return ji, ci, (r.status.copy(), r.ncomp.copy(), r.count1.copy(), r.comp_size.copy(), r.xy.copy())


@pytest.mark.parametrize("lanes", [2, 3])
def test_contexts_in_threads_match_one_context(lanes):
    import torch
    import gcmfgh
    base, ovl = synth.small_join(8, 4000)
    db, do = gcmfgh.DeviceLayer(base), gcmfgh.DeviceLayer(ovl)
    ref_eng = gcmfgh.Engine(0)
    try:
        ref = _result(ref_eng, db, do)
    finally:
        ref_eng.close()
    engines = [gcmfgh.Engine(0) for _ in range(lanes)]
    streams = [torch.cuda.Stream() for _ in range(lanes)]
    for e, st in zip(engines, streams):
        e.set_stream(st.cuda_stream)
    out = [[] for _ in range(lanes)]
    errs = []

    def worker(j):
        try:
            for _ in range(3):
                out[j].append(_result(engines[j], db, do))
        except Exception as e:
            errs.append(e)
    th = [threading.Thread(target=worker, args=(j,)) for j in range(lanes)]
    try:
        for t in th:
            t.start()
        for t in th:
            t.join()
    finally:
        for e in engines:
            e.close()
    assert not errs
    for runs in out:
        assert len(runs) == 3
        for ji, ci, arrays in runs:
            assert ji == ref[0] and ci == ref[1]
            for a, b in zip(arrays, ref[2]):
                assert np.array_equal(a, b)
