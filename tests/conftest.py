"""Shared fixtures: paths, the `gpu` marker, the engine (GPU) and the oracle (CPU)."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "gcmf-gh_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def build_library():
    lib = os.path.join(ROOT, "gcmf-gh_b200", "lib", "libgcmfgh.so")
    shims = os.path.join(ROOT, "gcmf-gh_b200", "lib", "libgcmfgh_shims.so")
    if not os.path.exists(lib) or not os.path.exists(shims):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "gcmf-gh_b200")], check=True)
    return lib


@pytest.fixture(scope="session")
def engine():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    build_library()
    import gcmfgh
    eng = gcmfgh.Engine(0)
    yield eng
    eng.close()


def load_poly(path):
    """Reference .poly text: 'x y,' per vertex, ';' closes a component."""
    comps = []
    for chunk in open(path).read().split(";"):
        v = chunk.replace(",", " ").split()
        if v:
            comps.append(np.array(v, dtype=np.float64).reshape(-1, 2))
    return comps


def format_reference(components):
    """The reference's output text (polygon.h:575-584 with ostream's default precision)."""
    out = []
    for c in components:
        lines = [f"{x:g} {y:g}" for x, y in c]
        out.append(",\n".join(lines) + ";\n")
    return "".join(out)


def same_components(a, b):
    return len(a) == len(b) and all(x.shape == y.shape and np.array_equal(x, y) for x, y in zip(a, b))


def unpack_pairs(path):
    d = np.load(path)
    nP, nQ, ncomp, csz = d["nP"], d["nQ"], d["ncomp"], d["comp_size"]
    P, Q, xy = d["P"], d["Q"], d["xy"]
    pairs, results = [], []
    op = oq = oc = ov = 0
    for k in range(len(nP)):
        pairs.append((P[2 * op:2 * (op + nP[k])].reshape(-1, 2), Q[2 * oq:2 * (oq + nQ[k])].reshape(-1, 2)))
        op += nP[k]
        oq += nQ[k]
        comps = []
        for _ in range(ncomp[k]):
            comps.append(xy[2 * ov:2 * (ov + csz[oc])].reshape(-1, 2))
            ov += csz[oc]
            oc += 1
        results.append(comps)
    return pairs, results


def unpack_multi(path):
    """(pairs, intersection results, union results) of a multi-component fixture made by
    tests/golden/make_multi_goldens.py; a pair is (P rings, Q rings)."""
    d = np.load(path)
    pairs, res = [], {"i_": [], "u_": []}
    si = so = 0
    for k in range(len(d["kP"])):
        sides = []
        for cnt in (d["kP"][k], d["kQ"][k]):
            rings = []
            for _ in range(cnt):
                m = int(d["sizes"][si])
                rings.append(d["xy"][2 * so:2 * (so + m)].reshape(-1, 2))
                si += 1
                so += m
            sides.append(rings)
        pairs.append(tuple(sides))
    for tag in res:
        oc = ov = 0
        for k in range(len(d["kP"])):
            comps = []
            for _ in range(int(d[tag + "ncomp"][k])):
                m = int(d[tag + "comp_size"][oc])
                comps.append(d[tag + "xy"][2 * ov:2 * (ov + m)].reshape(-1, 2))
                oc += 1
                ov += m
            res[tag].append(comps)
    return pairs, res["i_"], res["u_"]
