"""The C-ABI library loads without a GPU and exports what include/gisspa.h declares."""
import os
import re
import subprocess

import pytest

import gisspa_b200 as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "gisspa.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gs_[a-z_0-9]+)\s*\(", src)))


def test_header_matches_python_binding():
    assert sorted(G.EXPORTS) == _declared()


def test_library_exports_every_declared_symbol():
    if not os.path.exists(G.LIB_PATH):
        from gisspa_b200 import build
        build.build_library()
    out = subprocess.run(["nm", "-D", "--defined-only", G.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (gs_\w+)", out))
    missing = [s for s in _declared() if s not in exported]
    assert not missing, missing
    lib = G.load_library()
    for s in _declared():
        assert hasattr(lib, s)


def test_status_strings_and_defaults_without_gpu():
    lib = G.load_library()
    assert lib.gs_status_string(0) == b"ok"
    assert lib.gs_status_string(5) == b"unsupported input"
    p = G.default_params()
    # DataReader.h:16-42
    assert p.window_size == 320 and p.overlap == -1 and abs(p.thres - 7.0) < 1e-6
    assert p.apix == -1 and p.norm_type == 0 and abs(p.ampconst - 0.07) < 1e-7


def test_driver_help_runs_without_gpu():
    if not os.path.exists(G.DRIVER_PATH):
        from gisspa_b200 import build
        build.build_library()
        build.build_driver()
    r = subprocess.run([G.DRIVER_PATH, "-h"], capture_output=True, text=True)
    assert r.returncode == 0 and "config" in r.stdout
