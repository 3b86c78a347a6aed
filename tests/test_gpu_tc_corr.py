"""Tensor-core correlation (tccorr.cuh: N2-point DFT stage as a split
16-bit tcgen05 GEMM, FP32 accumulation) against the FP64 oracle, the FP32
CUDA path and the reference's own output.

Tolerances: scores within 1e-3 relative of the oracle (the bound stated for
the tensor-core path; the observed error is printed), identical peak
positions, identical picks except lines whose score lies within 1e-3 of the
threshold."""
import os

import numpy as np
import pytest

import _helpers as H
import gisspa_b200 as G
from gisspa_b200 import formats, synth
from oracle import gisspa_oracle as O

pytestmark = pytest.mark.gpu

TC_RTOL = 1e-3
PRECISIONS = {"bf16": 1, "fp16": 2}


@pytest.fixture(scope="module", autouse=True)
def _built():
    from gisspa_b200 import build
    build.build_library()


def _in_dir(d, fn, *a, **kw):
    cwd = os.getcwd()
    os.chdir(d)
    try:
        return fn(*a, **kw)
    finally:
        os.chdir(cwd)


@pytest.mark.parametrize("prec", sorted(PRECISIONS))
@pytest.mark.parametrize("l,overlap", [(720, 200), (768, 256), (512, 100)])
def test_tc_sizes_match_oracle(l, overlap, prec):
    ds = synth.make_dataset(21 + l, nx=int(l * 1.9), ny=int(l * 1.3), n_templates=3, tsize=110,
                            n_particles=3, snr=0.3, n_blobs=60, ball_radius=35.0, phistep=120.0,
                            diameter=100.0, window=l, overlap=overlap, defocus=(1.0, 2.0),
                            astig_A=300.0)
    m = ds.micrographs[0]
    p = O.Params(apix=1.0, phi_step=120.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=100.0,
                 d_m=100.0, thres=0.0, padding_size=l, phase_flip=1, overlap=overlap)
    ref = O.search(m.image, ds.templates, p, O.make_ctf(p, m.defocus, m.dfdiff, m.dfang, l),
                   workers=4)
    gp = G.default_params(apix=1.0, phi_step=120.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0,
                          lowres=100.0, d_m=100.0, thres=0.0, window_size=l, overlap=overlap,
                          phase_flip=1, precision=PRECISIONS[prec])
    with G.Context(0) as ctx:
        ctx.set_templates(gp, ds.templates, (m.defocus, m.dfdiff, m.dfang))
        ctx.search(m.image, (m.defocus, m.dfdiff, m.dfang))
        u = ctx.units(ref.score.shape)
    fin = np.isfinite(ref.score)
    assert np.array_equal(fin, np.isfinite(u["score"]))
    rel = np.abs(u["score"][fin] - ref.score[fin]) / np.abs(ref.score[fin])
    print("tc %s l=%d: max rel score error vs FP64 oracle %.3e over %d units"
          % (prec, l, rel.max(), fin.sum()))
    assert rel.max() <= TC_RTOL, rel.max()
    assert np.array_equal(u["pos"][fin], ref.pos[fin])


@pytest.mark.parametrize("prec", sorted(PRECISIONS))
def test_tc_bench_small_matches_reference_and_fp32(prec, tmp_path):
    """The 1024^2 / 50 templates / 72 angles / l = 512 workload: every unit
    against the FP32 path, every reference line reproduced."""
    H.materialize("bench_small", str(tmp_path))
    cfg = formats.read_config(str(tmp_path / "config"))
    ent = formats.read_lst_entry(str(tmp_path / cfg.inlst), 0)
    img = formats.read_mrc(ent.path, 0)
    stack = formats.read_mrc(str(tmp_path / cfg.temp2d), -1)
    ctf = (ent.defocus, ent.dfdiff, ent.dfang)
    out = {}
    for mode in (0, PRECISIONS[prec]):
        gp = G.params_from_config(cfg)
        gp.precision = mode
        with G.Context(0) as ctx:
            ctx.set_templates(gp, stack, ctf)
            picks = ctx.search(img, ctf)
            out[mode] = (ctx.units(), picks)
    (a, pa), (b, pb) = out[0], out[PRECISIONS[prec]]
    fin = np.isfinite(a["score"])
    assert np.array_equal(fin, np.isfinite(b["score"]))
    rel = np.abs(b["score"][fin] - a["score"][fin]) / np.abs(a["score"][fin])
    npos = int((a["pos"] != b["pos"])[fin].sum())
    print("tc %s vs fp32 on bench_small: max rel %.3e, %d of %d peak positions differ"
          % (prec, rel.max(), npos, fin.sum()))
    assert rel.max() <= TC_RTOL
    # a peak may move only between near-equal pixels (a tie within rounding):
    # at most 1 in 10^4 units, and those keep their score; the picks
    # themselves are compared with the reference's lines below
    diff = (a["pos"] != b["pos"]) & fin
    assert npos <= max(2, fin.sum() // 10000), npos
    if npos:
        assert rel[diff[fin]].max() <= 1e-4
    # reference lines, through the Python mirror of the driver
    gold = H.load_golden("bench_small")
    lines = [x.rstrip("\n") for x in _in_dir(str(tmp_path), G.run_config, "config",
                                              precision=PRECISIONS[prec])]
    r = H.compare_lines(gold["lines"], lines, 6.0, rtol=TC_RTOL)
    assert not r["bad_ref"] and not r["bad_got"], (r["bad_ref"][:3], r["bad_got"][:3])
    assert r["max_rel"] <= TC_RTOL
    assert r["n_ref"] > 4000
    print("tc %s vs reference lines: %d matched of %d, max rel %.3e"
          % (prec, r["matched"], r["n_ref"], r["max_rel"]))


def test_tc_refuses_unsupported_windows():
    gp = G.default_params(apix=1.0, phi_step=90.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0,
                          lowres=100.0, d_m=48.0, thres=0.0, window_size=128, overlap=32,
                          phase_flip=1, precision=1)
    ds = synth.make_dataset(3, nx=400, ny=352, n_templates=2, tsize=56, n_particles=1, snr=0.3,
                            n_blobs=20, ball_radius=16.0, phistep=90.0, diameter=48.0, window=128,
                            overlap=32)
    m = ds.micrographs[0]
    with G.Context(0) as ctx:
        ctx.set_templates(gp, ds.templates, (m.defocus, m.dfdiff, m.dfang))
        with pytest.raises(G.GisspaError) as e:
            ctx.search(m.image, (m.defocus, m.dfdiff, m.dfang))
        assert e.value.status == 5
