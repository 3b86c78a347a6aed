"""Golden vectors from the reference itself.

Generates the seeded synthetic cases below, runs the reference GisSPA binary
(built from the reference's own sources by ``oracle/Makefile`` into
``oracle/_ref/gisspa_ref``) on each of them on a GPU, and stores the
reference's output pick lines plus a SHA-256 of the generated inputs in
``tests/golden/<case>.json.gz``.  The tests regenerate the inputs from the same
seed, check the digest, and compare the oracle (and the CUDA path) with the
reference's lines.

    python tests/golden/make_golden.py --out <dir>          # needs a GPU
    python tests/golden/make_golden.py --list               # case names

Every case respects the reference's own limits: window size a multiple of
32 and overlap >= 0 (its reductions assume l % 32 == 0, and overlap -1 can
leave its whole-image buffer smaller than the micrograph).
"""
from __future__ import annotations

import argparse
import gzip
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from gisspa_b200 import synth  # noqa: E402

# name -> (make_dataset kwargs, extra config keys)
CASES = {
    # all units emitted (threshold 0) so every (angle, window, template) score is pinned
    "small_pf1_all": (dict(seed=11, nx=512, ny=384, n_templates=6, tsize=64, n_particles=4,
                           snr=0.3, n_blobs=60, ball_radius=20.0, phistep=30.0, diameter=48.0,
                           window=128, overlap=32, hot_pixels=5, threshold=0.0),
                      {}),
    "small_pf0_invert_astig": (dict(seed=12, nx=448, ny=512, n_templates=5, tsize=64,
                                    n_particles=4, snr=0.3, n_blobs=60, ball_radius=20.0,
                                    phistep=45.0, diameter=40.0, window=128, overlap=48,
                                    defocus=(1.2, 2.2), astig_A=400.0, phase_flip=0, invert=1,
                                    threshold=0.0),
                               {}),
    "small_astig_pf1_all": (dict(seed=13, nx=400, ny=416, n_templates=4, tsize=48,
                                 n_particles=3, snr=0.4, n_blobs=40, ball_radius=15.0,
                                 phistep=40.0, diameter=36.0, window=96, overlap=16,
                                 defocus=(0.9, 1.9), astig_A=450.0, noise_alpha=0.5,
                                 threshold=0.0, apix=1.3),
                            {}),
    # window smaller than the template: the reference rounds it up to 32*k
    "pad_adjust_two_mics": (dict(seed=14, nx=384, ny=384, n_templates=3, tsize=70,
                                 n_particles=3, snr=0.4, n_blobs=50, ball_radius=22.0,
                                 phistep=60.0, diameter=50.0, window=64, overlap=20,
                                 defocus=(1.0, 2.0), astig_A=300.0, n_micrographs=2,
                                 threshold=4.0),
                            {}),
    # norm_type 1: per-pixel z-scores over all templates and angles, 1024-element blocks
    "norm1_small": (dict(seed=15, nx=448, ny=384, n_templates=5, tsize=64, n_particles=3,
                         snr=0.4, n_blobs=60, ball_radius=20.0, phistep=45.0, diameter=48.0,
                         window=128, overlap=32, threshold=3.4),
                    {"norm_type": 1}),
    # norm_type 1 at a window of 512 = 16 x 32 (the specialised FFT kernels)
    "norm1_fast512": (dict(seed=16, nx=1100, ny=960, n_templates=5, tsize=120, n_particles=4,
                           snr=0.4, n_blobs=80, ball_radius=36.0, phistep=45.0, diameter=100.0,
                           window=512, overlap=100, threshold=3.6),
                      {"norm_type": 1}),
    # the small benchmark workload itself (1024^2, 50 x 128^2 templates, 72 angles)
    "bench_small": (dict(synth.config_small(seed=0)), {"threshold": 6.0}),
}


def case_dataset(name: str):
    kw, extra = CASES[name]
    kw = dict(kw)
    seed = kw.pop("seed")
    ds = synth.make_dataset(seed, **kw)
    return ds, extra


def dataset_digest(ds) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(ds.templates, dtype="<f4").tobytes())
    h.update(np.ascontiguousarray(ds.views, dtype="<f4").tobytes())
    for m in ds.micrographs:
        h.update(np.ascontiguousarray(m.image, dtype="<f4").tobytes())
        h.update(np.asarray([m.defocus, m.dfdiff, m.dfang], dtype="<f8").tobytes())
    return h.hexdigest()


def run_reference(binary: str, name: str, workdir: str) -> dict:
    ds, extra = case_dataset(name)
    d = os.path.join(workdir, name)
    cfg = synth.write_dataset(ds, d, extra)
    t0 = time.time()
    proc = subprocess.run([binary, "config"], cwd=d, capture_output=True, text=True,
                          timeout=1800)
    dt = time.time() - t0
    with open(os.path.join(d, "picks.lst")) as fh:
        lines = fh.read().splitlines()
    with open(cfg) as fh:
        config_text = fh.read()
    return {"case": name, "digest": dataset_digest(ds), "returncode": proc.returncode,
            "wall_s": dt, "config": config_text, "lines": lines}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=None, help="directory for the <case>.json.gz files")
    ap.add_argument("--binary", default=os.path.join(ROOT, "oracle", "_ref", "gisspa_ref"))
    ap.add_argument("--cases", nargs="*", default=list(CASES))
    ap.add_argument("--list", action="store_true")
    a = ap.parse_args()
    if a.list:
        print("\n".join(CASES))
        return 0
    if not a.out:
        ap.error("--out is required")
    os.makedirs(a.out, exist_ok=True)
    work = tempfile.mkdtemp(prefix="gisspa_golden_")
    rc = 0
    try:
        for name in a.cases:
            res = run_reference(a.binary, name, work)
            with gzip.open(os.path.join(a.out, name + ".json.gz"), "wt") as fh:
                json.dump(res, fh)
            print("%s: rc=%d lines=%d wall=%.1fs" % (name, res["returncode"], len(res["lines"]),
                                                     res["wall_s"]))
            rc |= res["returncode"]
    finally:
        shutil.rmtree(work, ignore_errors=True)
    return rc


if __name__ == "__main__":
    sys.exit(main())
