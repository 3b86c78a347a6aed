"""The oracle against the reference's own outputs (golden vectors).

The fixtures in tests/golden/ were produced by the reference GisSPA binary,
built from its own sources (oracle/Makefile) and run on a B200, on seeded
synthetic inputs that the tests regenerate.  Every discrete field of every
output line (micrograph, path, CTF values, Euler angles, centre) must match
exactly, and scores to float32 noise."""
import os

import pytest

import _helpers as H
from oracle import gisspa_oracle as O


def _run_oracle(name, tmp_path):
    cfg, _ = H.materialize(name, str(tmp_path))
    cwd = os.getcwd()
    os.chdir(str(tmp_path))
    try:
        return O.run_config("config", workers=4)
    finally:
        os.chdir(cwd)


@pytest.mark.parametrize("name", H.SMALL_CASES + H.NORM1_CASES)
def test_oracle_matches_reference(name, tmp_path):
    gold = H.load_golden(name)
    assert gold["returncode"] == 0
    lines = [l.rstrip("\n") for l in _run_oracle(name, tmp_path)]
    thres = float([l for l in gold["config"].splitlines() if l.startswith("threshold")][0].split("=")[1])
    r = H.compare_lines(gold["lines"], lines, thres, rtol=1e-5)
    assert r["n_ref"] == len(gold["lines"]) and r["n_ref"] > 50
    assert not r["bad_ref"] and not r["bad_got"], (r["bad_ref"][:3], r["bad_got"][:3])
    assert r["matched"] == r["n_ref"] == r["n_got"]
    assert r["max_rel"] < 1e-5
    # same line order as the reference
    assert [l.split("\tscore=")[0] for l in lines] == [l.split("\tscore=")[0] for l in gold["lines"]]


@pytest.mark.slow
@pytest.mark.skipif(os.environ.get("GISSPA_SLOW") != "1", reason="set GISSPA_SLOW=1 (several minutes)")
def test_oracle_matches_reference_bench_small(tmp_path):
    gold = H.load_golden("bench_small")
    lines = [l.rstrip("\n") for l in _run_oracle("bench_small", tmp_path)]
    r = H.compare_lines(gold["lines"], lines, 6.0, rtol=1e-5)
    assert not r["bad_ref"] and not r["bad_got"]
    assert r["max_rel"] < 1e-5
