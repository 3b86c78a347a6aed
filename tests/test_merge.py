"""Duplicate merging (the reference's remove_repeat_particles_from_list.py):
the oracle restatement against the script's own outputs
(tests/golden/merge_cases.json.gz, made by tests/golden/make_merge_golden.py
from the unchanged script), and the merging path on the GPU (library and
drop-in CLI) against the same outputs."""
import gzip
import json
import os
import subprocess

import pytest

import _helpers as H
from oracle import merge_oracle as M


def _cases():
    with gzip.open(os.path.join(H.GOLDEN, "merge_cases.json.gz"), "rt") as fh:
        return json.load(fh)["cases"]


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c["name"])
def test_oracle_matches_script(case):
    out = M.merge_lines(case["input"], case["center"], case["euler_thres"])
    assert out == case["output"]
    assert len(out) < len(case["input"])


@pytest.mark.gpu
@pytest.mark.parametrize("case", _cases(), ids=lambda c: c["name"])
def test_gpu_merge_matches_script(case):
    import gisspa_b200 as G
    from gisspa_b200 import build
    build.build_library()
    out = G.merge_lines(case["input"], case["center"], case["euler_thres"])
    assert out == case["output"]


@pytest.mark.gpu
def test_merge_cli_matches_script(tmp_path):
    import gisspa_b200 as G
    from gisspa_b200 import build
    build.build_library()
    build.build_merge_cli()
    for case in _cases():
        inp, out = tmp_path / "in.lst", tmp_path / "out.lst"
        inp.write_text("".join(case["input"]))
        r = subprocess.run([G.MERGE_CLI_PATH, str(inp), "64", str(case["center"]),
                            str(case["euler_thres"]), str(out)], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        assert out.read_text() == "".join(case["output"]), case["name"]
