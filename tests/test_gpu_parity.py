"""CUDA path (through the C ABI) against the FP64 oracle and the reference.

* every (angle, window, template) unit: score within 1e-4 relative of the
  oracle, identical peak position;
* every output line against the reference's own output (golden vectors):
  identical discrete fields, scores within 1e-4 relative; a line may only be
  missing on one side when its score is within 1e-4 of the threshold.
"""
import os

import numpy as np
import pytest

import _helpers as H
import gisspa_b200 as G
from gisspa_b200 import formats
from oracle import gisspa_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    from gisspa_b200 import build
    build.build_library()
    build.build_driver()


def _in_dir(d, fn, *a, **kw):
    cwd = os.getcwd()
    os.chdir(d)
    try:
        return fn(*a, **kw)
    finally:
        os.chdir(cwd)


@pytest.mark.parametrize("name", H.SMALL_CASES)
def test_lines_match_reference(name, tmp_path):
    H.materialize(name, str(tmp_path))
    gold = H.load_golden(name)
    lines = [l.rstrip("\n") for l in _in_dir(str(tmp_path), G.run_config, "config")]
    cfg = formats.read_config(str(tmp_path / "config"))
    r = H.compare_lines(gold["lines"], lines, cfg.thres)
    assert not r["bad_ref"] and not r["bad_got"], (r["bad_ref"][:3], r["bad_got"][:3])
    assert r["max_rel"] <= H.SCORE_RTOL, r["max_rel"]
    assert r["matched"] >= r["n_ref"] - len(r["only_ref"])


@pytest.mark.parametrize("name", H.SMALL_CASES)
def test_units_match_oracle(name, tmp_path):
    H.materialize(name, str(tmp_path))
    lines, tables = _in_dir(str(tmp_path), G.run_config, "config", return_units=True)
    _, results = _in_dir(str(tmp_path), O.run_config, "config", workers=4, return_results=True)
    assert len(tables) == len(results)
    for tab, res in zip(tables, results):
        so, sg = res.score, tab["score"].astype(np.float64)
        assert so.shape == sg.shape
        fin = np.isfinite(so)
        assert np.array_equal(fin, np.isfinite(sg))
        rel = np.abs(sg[fin] - so[fin]) / np.maximum(np.abs(so[fin]), 1e-6)
        assert rel.max() <= H.SCORE_RTOL, rel.max()
        pos_bad = (tab["pos"] != res.pos) & fin
        assert pos_bad.sum() == 0, np.argwhere(pos_bad)[:5]
        pk = np.abs(tab["peak"] - res.peak) / np.maximum(np.abs(res.peak), 1e-12)
        assert pk.max() <= H.SCORE_RTOL


@pytest.mark.parametrize("name", ["small_pf1_all"])
def test_driver_matches_reference(name, tmp_path):
    import subprocess
    H.materialize(name, str(tmp_path))
    r = subprocess.run([G.DRIVER_PATH, "config"], cwd=str(tmp_path), capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    got = (tmp_path / "picks.lst").read_text().splitlines()
    gold = H.load_golden(name)
    res = H.compare_lines(gold["lines"], got, 0.0)
    assert not res["bad_ref"] and not res["bad_got"]
    assert res["max_rel"] <= H.SCORE_RTOL


def test_search_device_equals_host_path(tmp_path):
    torch = pytest.importorskip("torch")
    H.materialize("small_pf1_all", str(tmp_path))
    cfg = formats.read_config(str(tmp_path / "config"))
    ent = formats.read_lst_entry(str(tmp_path / cfg.inlst), 0)
    img = formats.read_mrc(ent.path, 0)
    stack = formats.read_mrc(str(tmp_path / cfg.temp2d), -1)
    with G.Context(0) as ctx:
        ctx.set_templates(G.params_from_config(cfg), stack, (ent.defocus, ent.dfdiff, ent.dfang))
        a = ctx.search(img, (ent.defocus, ent.dfdiff, ent.dfang))
        d = torch.from_numpy(img).cuda()
        torch.cuda.synchronize()
        b = ctx.search_device(d.data_ptr(), img.shape[1], img.shape[0], (ent.defocus, ent.dfdiff, ent.dfang))
        assert np.array_equal(a, b)
        assert np.array_equal(d.cpu().numpy(), img)   # input untouched
