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


def test_header_constants_match_python_binding():
    """Every GS_OPT_* and GS_PREC_* value the header defines is the Python
    module's constant of the same name."""
    src = open(os.path.join(ROOT, "include", "gisspa.h")).read()
    defs = dict(re.findall(r"^#define (GS_(?:OPT|PREC)_[A-Z0-9_]+) (\d+)\s*$", src, flags=re.M))
    assert len(defs) >= 15, defs
    for name, value in defs.items():
        assert getattr(G, name) == int(value), name


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


_HAS_GPU_DEVICE = os.path.exists("/dev/nvidiactl") or os.path.exists("/dev/nvidia0")


@pytest.mark.skipif(_HAS_GPU_DEVICE, reason="a GPU is present: the no-GPU failure path cannot be shown here")
def test_no_gpu_is_an_error_not_a_fallback(tmp_path):
    # without a CUDA device the library refuses to work (no CPU fallback):
    # context creation returns GS_ERR_CUDA, the Python binding raises, and the
    # drop-in driver exits non-zero after reading its inputs
    import ctypes as C
    import _helpers as H
    lib = G.load_library()
    h = C.c_void_p()
    assert lib.gs_ctx_create(0, C.byref(h)) == G.GS_ERR_CUDA
    with pytest.raises(G.GisspaError) as e:
        G.Context(0)
    assert e.value.status == G.GS_ERR_CUDA
    if not os.path.exists(G.DRIVER_PATH):
        from gisspa_b200 import build
        build.build_driver()
    H.materialize("small_pf1_all", str(tmp_path))
    r = subprocess.run([G.DRIVER_PATH, "config"], cwd=str(tmp_path), capture_output=True, text=True,
                       timeout=300)
    assert r.returncode != 0
    assert "CUDA" in r.stderr or "cuda" in r.stderr
    assert not (tmp_path / "picks.lst").exists() or (tmp_path / "picks.lst").read_text() == ""


def test_header_is_plain_c(tmp_path):
    # a C caller (the way a reference-side program would bind the library)
    # compiles and links against include/gisspa.h with strict C99
    import shutil
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    if not os.path.exists(G.LIB_PATH):
        from gisspa_b200 import build
        build.build_library()
    src = tmp_path / "caller.c"
    src.write_text(
        '#include "gisspa.h"\n'
        "int main(void) {\n"
        "    gs_ctx* ctx = 0;\n"
        "    gs_params p;\n"
        "    float* img = 0; int nx, ny, nz; char err[64];\n"
        "    gs_params_default(&p);\n"
        "    if (gs_ctx_create(0, &ctx) == GS_OK) gs_ctx_destroy(ctx);\n"
        "    if (gs_hdf_read_image(\"x.hdf\", 0, &img, &nx, &ny, &nz, err, sizeof err) == GS_OK) gs_host_free(img);\n"
        "    return 0;\n"
        "}\n")
    libdir = os.path.dirname(G.LIB_PATH)
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror",
                        "-I" + os.path.join(ROOT, "include"), str(src), "-L" + libdir, "-lgisspa_b200",
                        "-Wl,-rpath," + libdir, "-o", str(tmp_path / "caller")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
