"""EMAN HDF5 inputs through the drop-in driver and its Python mirror.

The reference's golden case is re-run with its template stack written as an
EMAN2 file (/MDF/images/<n>/image) and its micrograph as an old-style EMAN
file (root dataset "<nn>", nx = dims[0]); both readers must hand the search the
same pixels as the MRC inputs, so the output lines must match the reference's
own output for the MRC inputs (paths aside) as the MRC run does.
"""
import os
import subprocess

import pytest

import _hdf5_writer as W
import _helpers as H
import gisspa_b200 as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    from gisspa_b200 import build
    build.build_library()
    build.build_driver()


def test_hdf_inputs_reproduce_reference_lines(tmp_path):
    name = "small_pf1_all"
    H.materialize(name, str(tmp_path))
    W.copy_case_as_hdf(str(tmp_path))
    gold = H.load_golden(name)
    cwd = os.getcwd()
    os.chdir(str(tmp_path))
    try:
        py_lines = [l.rstrip("\n") for l in G.run_config("config_hdf")]
    finally:
        os.chdir(cwd)
    r = subprocess.run([G.DRIVER_PATH, "config_hdf"], cwd=str(tmp_path), capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    drv_lines = (tmp_path / "picks.lst").read_text().splitlines()
    assert drv_lines and all(".hdf" in l for l in drv_lines)
    for got in (py_lines, drv_lines):
        got = [l.replace(".hdf", ".mrc") for l in got]
        res = H.compare_lines(gold["lines"], got, 0.0)
        assert not res["bad_ref"] and not res["bad_got"], (res["bad_ref"][:3], res["bad_got"][:3])
        assert res["max_rel"] <= H.SCORE_RTOL, res["max_rel"]

