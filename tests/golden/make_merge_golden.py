"""Golden vectors for duplicate merging, produced by the reference's own
script (python_scripts/remove_repeat_particles_from_list.py).

The script is Python 2; it is run here unchanged except for two mechanical
steps that Python 3 needs to compile it: tabs are expanded to 8 columns (how
Python 2 reads its mixed indentation) and its one `print` statement (in the
usage message, never reached here) becomes a call.  Inputs are real pick
lists: the reference's own output lines of the golden search cases, several
micrographs concatenated, at several centre / Euler thresholds.

    python tests/golden/make_merge_golden.py --reference <reference checkout>

writes tests/golden/merge_cases.json.gz.
"""
from __future__ import annotations

import argparse
import gzip
import json
import os
import re
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))

SCRIPT = os.path.join("python_scripts", "remove_repeat_particles_from_list.py")

# (name, golden search cases whose lines form the input, centre threshold px, Euler threshold deg)
CASES = [
    ("bench_small_c45_e15", ["bench_small"], 45.0, 15.0),
    ("bench_small_c20_e40", ["bench_small"], 20.0, 40.0),
    ("two_mics_c30_e10", ["pad_adjust_two_mics", "small_astig_pf1_all"], 30.0, 10.0),
    ("norm1_c24_e20", ["norm1_small", "small_pf1_all"], 24.0, 20.0),
]


def load_reference_main(ref_root: str):
    src = open(os.path.join(ref_root, SCRIPT)).read().expandtabs(8)
    src = re.sub(r'print\s+"([^"]*)"', r'print("\1")', src)
    ns = {"__name__": "reference_merge"}
    exec(compile(src, SCRIPT, "exec"), ns)
    return ns["main"]


def golden_lines(name: str):
    with gzip.open(os.path.join(HERE, name + ".json.gz"), "rt") as fh:
        g = json.load(fh)
    return [l if l.endswith("\n") else l + "\n" for l in g["lines"]]


def run_case(main, lines, center, euler):
    with tempfile.TemporaryDirectory() as d:
        inp, out = os.path.join(d, "in.lst"), os.path.join(d, "out.lst")
        with open(inp, "w") as fh:
            fh.writelines(lines)
        argv = sys.argv
        sys.argv = ["remove_repeat_particles_from_list.py", inp, "64", str(center), str(euler), out]
        try:
            main()
        finally:
            sys.argv = argv
        return open(out).read().splitlines(True)


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the reference checkout")
    ap.add_argument("--out", default=os.path.join(HERE, "merge_cases.json.gz"))
    args = ap.parse_args()
    ref_main = load_reference_main(args.reference)
    cases = []
    for name, sources, center, euler in CASES:
        lines = []
        for s in sources:
            lines += golden_lines(s)
        out = run_case(ref_main, lines, center, euler)
        cases.append({"name": name, "sources": sources, "center": center, "euler_thres": euler,
                      "input": lines, "output": out})
        print("%s: %d -> %d lines" % (name, len(lines), len(out)))
    with gzip.open(args.out, "wt") as fh:
        json.dump({"script": SCRIPT, "cases": cases}, fh)
    return 0


if __name__ == "__main__":
    sys.exit(main())
