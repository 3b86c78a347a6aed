"""Specialised l = 16*N2 kernels (l = 512, 720, 768) against the reference,
the oracle and the generic kernels."""
import os

import numpy as np
import pytest

import _helpers as H
import gisspa_b200 as G
from gisspa_b200 import formats, synth
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


def test_bench_small_lines_match_reference(tmp_path):
    """The 1024^2 / 50 templates / 72 angles / l = 512 workload through the
    fast kernels: every reference line reproduced."""
    H.materialize("bench_small", str(tmp_path))
    gold = H.load_golden("bench_small")
    lines = [l.rstrip("\n") for l in _in_dir(str(tmp_path), G.run_config, "config")]
    r = H.compare_lines(gold["lines"], lines, 6.0)
    assert not r["bad_ref"] and not r["bad_got"], (r["bad_ref"][:3], r["bad_got"][:3])
    assert r["max_rel"] <= H.SCORE_RTOL
    assert r["matched"] >= r["n_ref"] - len(r["only_ref"]) and r["n_ref"] > 4000


def test_fast_equals_generic_kernels(tmp_path):
    H.materialize("bench_small", str(tmp_path))
    cfg = formats.read_config(str(tmp_path / "config"))
    ent = formats.read_lst_entry(str(tmp_path / cfg.inlst), 0)
    img = formats.read_mrc(ent.path, 0)
    stack = formats.read_mrc(str(tmp_path / cfg.temp2d), -1)
    ctf = (ent.defocus, ent.dfdiff, ent.dfang)
    tabs = []
    for generic in (False, True):
        with G.Context(0) as ctx:
            ctx.set_generic_fft(generic)
            ctx.set_templates(G.params_from_config(cfg), stack, ctf)
            ctx.search(img, ctf)
            tabs.append(ctx.units())
    a, b = tabs
    fin = np.isfinite(a["score"])
    assert np.array_equal(fin, np.isfinite(b["score"]))
    rel = np.abs(a["score"][fin] - b["score"][fin]) / np.abs(b["score"][fin])
    assert rel.max() < 2e-5, rel.max()
    assert (a["pos"] != b["pos"]).sum() <= 2


@pytest.mark.parametrize("l,overlap", [(720, 200), (768, 256), (512, 100)])
def test_fast_sizes_match_oracle(l, overlap):
    ds = synth.make_dataset(21 + l, nx=int(l * 1.9), ny=int(l * 1.3), n_templates=3, tsize=110,
                            n_particles=3, snr=0.3, n_blobs=60, ball_radius=35.0, phistep=120.0,
                            diameter=100.0, window=l, overlap=overlap, defocus=(1.0, 2.0),
                            astig_A=300.0)
    m = ds.micrographs[0]
    p = O.Params(apix=1.0, phi_step=120.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=100.0,
                 d_m=100.0, thres=0.0, padding_size=l, phase_flip=1, overlap=overlap)
    ctf = O.make_ctf(p, m.defocus, m.dfdiff, m.dfang, l)
    ref = O.search(m.image, ds.templates, p, ctf, workers=4)
    gp = G.default_params(apix=1.0, phi_step=120.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0,
                          lowres=100.0, d_m=100.0, thres=0.0, window_size=l, overlap=overlap,
                          phase_flip=1)
    with G.Context(0) as ctx:
        ctx.set_templates(gp, ds.templates, (m.defocus, m.dfdiff, m.dfang))
        picks = ctx.search(m.image, (m.defocus, m.dfdiff, m.dfang))
        u = ctx.units(ref.score.shape)
    fin = np.isfinite(ref.score)
    assert np.array_equal(fin, np.isfinite(u["score"]))
    rel = np.abs(u["score"][fin] - ref.score[fin]) / np.abs(ref.score[fin])
    assert rel.max() <= H.SCORE_RTOL, rel.max()
    assert np.array_equal(u["pos"][fin], ref.pos[fin])
    assert len(picks) == len(ref.picks)


def test_persistent_equals_two_pass(tmp_path):
    """One persistent launch per angle (dependency-tracked row/column tiles,
    scratch ring) against per-window row and column launches, and against
    other unit orders (window blocks of 1 and 5)."""
    H.materialize("bench_small", str(tmp_path))
    cfg = formats.read_config(str(tmp_path / "config"))
    ent = formats.read_lst_entry(str(tmp_path / cfg.inlst), 0)
    img = formats.read_mrc(ent.path, 0)
    stack = formats.read_mrc(str(tmp_path / cfg.temp2d), -1)
    ctf = (ent.defocus, ent.dfdiff, ent.dfang)
    tabs = []
    for two_pass, block in ((True, 4), (False, 4), (False, 1), (False, 5)):
        with G.Context(0) as ctx:
            ctx.set_two_pass(two_pass)
            ctx.set_window_block(block)
            ctx.set_templates(G.params_from_config(cfg), stack, ctf)
            picks = ctx.search(img, ctf)
            tabs.append((ctx.units(), picks))
    ref, ref_picks = tabs[0]
    fin = np.isfinite(ref["score"])
    for u, picks in tabs[1:]:
        assert np.array_equal(fin, np.isfinite(u["score"]))
        rel = np.abs(u["score"][fin] - ref["score"][fin]) / np.abs(ref["score"][fin])
        assert rel.max() < 1e-6, rel.max()
        assert np.array_equal(u["pos"], ref["pos"])
        assert len(picks) == len(ref_picks)
