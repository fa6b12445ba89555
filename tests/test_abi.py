"""CPU checks of the C ABI: the library builds for sm_100a, loads, and exports every
function include/*.h declares.  No compute call is made (there is no GPU here)."""
import ctypes
import glob
import os
import re
import subprocess

from conftest import ROOT, build_library


def declared_functions(header="gcmfgh.h"):
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", header)):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"^\s*#.*$", "", text, flags=re.M)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;", text):
            name = m.group(1)
            if name not in {"if", "while", "for", "return", "sizeof"}:
                names.add(name)
    return names


def test_header_declares_the_entry_points():
    names = declared_functions()
    for n in ("gcmf_join", "gh_clip_batch", "gh_clip_pair", "gh_clip_joined", "gcmfgh_create",
              "gh_calculate_intersections", "gh_free_intersections",
              "gcmfgh_join_clip_host", "gcmfgh_exclusive_scan_i32", "gcmfgh_radix_sort_u64"):
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = build_library()
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = declared_functions() - exported
    assert not missing, missing


def test_shim_library_exports_the_reference_signatures():
    """include/gcmfgh_shims.h: C++ symbols whose mangled names equal the reference's
    declarations (main.h:5-11, coord_t = double), so its main.cpp links unchanged."""
    build_library()
    lib = os.path.join(ROOT, "gcmf-gh_b200", "lib", "libgcmfgh_shims.so")
    out = subprocess.run(["nm", "-DC", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    assert "spatialJoin(int, char**, int**, int**, long*, double**, double**, int**, long**, int**, long**)" in out
    assert "ghcuda(int*, int*, int, double*, double*, int*, long*, int*, long*)" in out
    assert ("calculateIntersections(double*, double*, int, int, double*, int*, long*, int*, long*, int, int, "
            "int*, int*, double**, double**, int**, int**, int**, int**, int**, int**, int*)") in out
    assert declared_functions("gcmfgh_shims.h") == {"spatialJoin", "ghcuda", "calculateIntersections"}


def test_library_loads_and_reports_status_strings():
    L = ctypes.CDLL(build_library())
    L.gcmfgh_status_string.restype = ctypes.c_char_p
    assert L.gcmfgh_status_string(0) == b"ok"
    assert L.gcmfgh_status_string(6) == b"destination too small"


def test_library_built_for_sm100a():
    lib = build_library()
    out = subprocess.run(["cuobjdump", "--list-elf", lib], capture_output=True, text=True).stdout
    assert "sm_100a" in out


def test_python_front_end_fails_loudly_without_library(tmp_path, monkeypatch):
    import gcmfgh
    monkeypatch.setattr(gcmfgh, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(gcmfgh, "_lib", None)
    try:
        gcmfgh.lib()
    except gcmfgh.GcmfghError:
        pass
    else:
        raise AssertionError("expected GcmfghError")
