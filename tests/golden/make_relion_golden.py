"""Golden vectors for the .lst -> RELION STAR export, produced by the
reference's own script (python_scripts/convert_my-lst_to_relion_mic.py).

The Python 2 script runs unchanged but for what Python 3 needs: tabs expanded
to 8 columns, its one `print` statement (usage message, not reached) made a
call, and Python 2's str() of floats (12 significant digits, '.0' added to
integral values) provided to it, since Python 3's str() prints differently.
Inputs are the reference's own pick lines of the golden search cases.

    python tests/golden/make_relion_golden.py --reference <reference checkout>
"""
from __future__ import annotations

import argparse
import builtins
import gzip
import json
import os
import re
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
SCRIPT = os.path.join("python_scripts", "convert_my-lst_to_relion_mic.py")

# (golden search case, scale, pixel size, micrographs dir, first lines used)
CASES = [("bench_small", 1, 1.0, "micrographs/", 600),
         ("pad_adjust_two_mics", 2, 1.34, "mics/", None),
         ("norm1_small", 3, 0.83, "", None)]


def _py2_str(x=""):
    if isinstance(x, float):
        s = "%.12g" % x
        if not any(c in s for c in ".en"):
            s += ".0"
        return s
    return builtins.str(x)


def load_reference_main(ref_root: str):
    src = open(os.path.join(ref_root, SCRIPT)).read().expandtabs(8)
    src = re.sub(r'print\s+"([^"]*)"', r'print("\1")', src)
    ns = {"__name__": "reference_relion", "str": _py2_str}
    exec(compile(src, SCRIPT, "exec"), ns)
    return ns["main"]


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True)
    ap.add_argument("--out", default=os.path.join(HERE, "relion_cases.json.gz"))
    args = ap.parse_args()
    ref_main = load_reference_main(args.reference)
    cases = []
    for name, scale, apix, mdir, first in CASES:
        with gzip.open(os.path.join(HERE, name + ".json.gz"), "rt") as fh:
            lines = [l if l.endswith("\n") else l + "\n" for l in json.load(fh)["lines"]][:first]
        with tempfile.TemporaryDirectory() as d:
            inp, out = os.path.join(d, "in.lst"), os.path.join(d, "out.star")
            open(inp, "w").writelines(lines)
            argv = sys.argv
            sys.argv = ["convert_my-lst_to_relion_mic.py", inp, str(scale), str(apix), out, mdir]
            try:
                ref_main()
            finally:
                sys.argv = argv
            star = open(out).read()
        cases.append({"name": name, "scale": scale, "apix": apix, "mdir": mdir, "input": lines,
                      "output": star})
        print("%s: %d lines -> %d bytes" % (name, len(lines), len(star)))
    with gzip.open(args.out, "wt") as fh:
        json.dump({"script": SCRIPT, "cases": cases}, fh)
    return 0


if __name__ == "__main__":
    sys.exit(main())
