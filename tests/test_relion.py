""".lst -> RELION STAR export against the reference script's own outputs
(tests/golden/relion_cases.json.gz, made by tests/golden/make_relion_golden.py),
through the function and the command line."""
import gzip
import json
import os
import subprocess
import sys

import pytest

import _helpers as H
from gisspa_b200 import relion


def _cases():
    with gzip.open(os.path.join(H.GOLDEN, "relion_cases.json.gz"), "rt") as fh:
        return json.load(fh)["cases"]


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c["name"])
def test_star_matches_script(case):
    assert relion.lst_to_star(case["input"], case["scale"], case["apix"], case["mdir"]) == case["output"]


def test_cli(tmp_path):
    case = _cases()[1]
    inp, out = tmp_path / "in.lst", tmp_path / "out.star"
    inp.write_text("".join(case["input"]))
    root = os.path.dirname(H.HERE)
    r = subprocess.run([sys.executable, "-m", "gisspa_b200.relion", str(inp), str(case["scale"]),
                        str(case["apix"]), str(out), case["mdir"]], cwd=root, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert out.read_text() == case["output"]


def test_py2_float_str():
    assert relion.py2_float_str(1.0) == "1.0"
    assert relion.py2_float_str(-270.0) == "-270.0"
    assert relion.py2_float_str(0.1 + 0.2) == "0.3"
    assert relion.py2_float_str(1e16) == "1e+16"
    assert relion.py2_float_str(12345.678901234) == "12345.6789012"
