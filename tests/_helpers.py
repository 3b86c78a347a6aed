"""Shared test helpers: golden cases (reference outputs) and comparisons."""
from __future__ import annotations

import gzip
import json
import os
import sys
from typing import Dict, List, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
sys.path.insert(0, GOLDEN)

import make_golden  # noqa: E402
from gisspa_b200 import formats, synth  # noqa: E402

SMALL_CASES = ["small_pf1_all", "small_pf0_invert_astig", "small_astig_pf1_all",
               "pad_adjust_two_mics"]
# norm_type 1 (per-pixel z-scores, 1024-element blocks)
NORM1_CASES = ["norm1_small", "norm1_fast512"]

# scores of the FP32 CUDA path against the FP64 oracle / the reference
SCORE_RTOL = 1e-4


def load_golden(name: str) -> dict:
    with gzip.open(os.path.join(GOLDEN, name + ".json.gz"), "rt") as fh:
        return json.load(fh)


def materialize(name: str, outdir: str) -> Tuple[str, object]:
    """Regenerate the case's inputs (checked against the stored digest) and
    write them with their config into ``outdir``; returns (config path, dataset)."""
    ds, extra = make_golden.case_dataset(name)
    gold = load_golden(name)
    assert make_golden.dataset_digest(ds) == gold["digest"], "synthetic inputs changed"
    cfg = synth.write_dataset(ds, outdir, extra)
    return cfg, ds


def compare_lines(ref: List[str], got: List[str], thres: float, rtol: float = SCORE_RTOL) -> Dict:
    """Match output lines by (nn, path, euler, template view, centre).

    A line present on one side only is tolerated when its score is within
    ``rtol`` of the threshold (it can flip across it by rounding)."""
    def key(d):
        return (d["nn"], d["path"], d["euler"], d["center"], d["defocus"], d["dfdiff"], d["dfang"])

    R = [formats.parse_pick_line(x) for x in ref]
    G = [formats.parse_pick_line(x) for x in got]
    rk = {}
    for i, d in enumerate(R):
        rk.setdefault(key(d), []).append(i)
    used = set()
    worst = 0.0
    only_got = []
    for d in G:
        lst = rk.get(key(d), [])
        hit = None
        for i in lst:
            if i not in used:
                hit = i
                break
        if hit is None:
            only_got.append(d)
            continue
        used.add(hit)
        worst = max(worst, abs(R[hit]["score"] - d["score"]) / max(abs(R[hit]["score"]), 1e-6))
    only_ref = [R[i] for i in range(len(R)) if i not in used]
    near = lambda d: abs(d["score"] - thres) <= rtol * max(abs(thres), 1.0) + 1e-6
    bad_ref = [d for d in only_ref if not near(d)]
    bad_got = [d for d in only_got if not near(d)]
    # order check: the matched lines must appear in the same relative order
    return {"n_ref": len(R), "n_got": len(G), "matched": len(used), "max_rel": worst,
            "only_ref": only_ref, "only_got": only_got, "bad_ref": bad_ref, "bad_got": bad_got}
