"""The reference's main() flow through the C++ shims (include/gcmfgh_shims.h): text
layers on disk -> spatialJoin -> ghcuda -> result file, compared with the oracle's join
and clip of the same files written in the reference's .poly format."""
import os
import subprocess

import numpy as np
import pytest

import pyoracle
from conftest import ROOT, format_reference
from gcmfgh import synth

pytestmark = pytest.mark.gpu


def test_reference_main_through_shims(tmp_path):
    import gcmfgh
    base, ovl = synth.small_join(0, 2000)
    fb, fo, fr = tmp_path / "base.txt", tmp_path / "overlay.txt", tmp_path / "result.poly"
    gcmfgh.write_text_layer(str(fb), base)
    gcmfgh.write_text_layer(str(fo), ovl)
    exe = tmp_path / "shim_main"
    lib = os.path.join(ROOT, "gcmf-gh_b200", "lib")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "shim_main.cpp"), "-o", str(exe), "-L", lib,
                    "-lgcmfgh_shims", f"-Wl,-rpath,{lib}"], check=True)
    env = dict(os.environ, GCMFGH_BASE_FILE=str(fb), GCMFGH_OVERLAY_FILE=str(fo), GCMFGH_RESULT_FILE=str(fr))
    subprocess.run([str(exe), "1", "x"], check=True, env=env, timeout=300)
    # the oracle on the same files, in the same order (clip set sorted by base, overlay)
    rb, _ = gcmfgh.read_text_layer(str(fb))
    ro, _ = gcmfgh.read_text_layer(str(fo))
    j = pyoracle.join(rb, ro)
    sel = j.clip == 1
    c = pyoracle.clip_batch(rb, ro, j.b[sel], j.o[sel])
    comps = []
    for k in range(int(sel.sum())):
        comps.extend(c.components(k))
    assert len(comps) > 100
    assert fr.read_text() == format_reference(comps)
