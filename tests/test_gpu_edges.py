"""Edge cases of the search on the GPU.

* window sizes that the specialised l = 16 N2 kernels do not cover go
  through the generic mixed-radix kernels: l = 160 (radices 8, 4, 5),
  208 (13 = a prime radix) and 224 (7), odd template counts, non-square
  micrographs whose whole-image FFTs have prime factors 11, 23 and 59:
  every unit against the oracle (score within 1e-4, same peak position);
* a threshold above every score gives no picks, and the drop-in driver then
  writes an empty output file;
* calls out of order and invalid parameters return their status codes and
  leave the context usable.
"""
import os
import subprocess

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


@pytest.mark.parametrize("l,nx,ny,nt", [(160, 418, 368, 3), (208, 506, 460, 5), (224, 472, 413, 4)])
def test_generic_window_sizes_match_oracle(l, nx, ny, nt):
    overlap = l // 4
    ds = synth.make_dataset(60 + l, nx=nx, ny=ny, n_templates=nt, tsize=64, n_particles=2, snr=0.4,
                            n_blobs=40, ball_radius=20.0, phistep=72.0, diameter=56.0, window=l,
                            overlap=overlap, defocus=(1.1, 1.9), astig_A=300.0)
    m = ds.micrographs[0]
    p = O.Params(apix=1.0, phi_step=72.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=100.0,
                 d_m=56.0, thres=0.0, padding_size=l, phase_flip=1, overlap=overlap)
    ref = O.search(m.image, ds.templates, p, O.make_ctf(p, m.defocus, m.dfdiff, m.dfang, l), workers=4)
    gp = G.default_params(apix=1.0, phi_step=72.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0,
                          lowres=100.0, d_m=56.0, thres=0.0, window_size=l, overlap=overlap, phase_flip=1)
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


def test_no_picks_and_empty_output(tmp_path):
    H.materialize("small_pf1_all", str(tmp_path))
    cfg = (tmp_path / "config").read_text().splitlines()
    cfg = [("threshold = 1000" if ln.startswith("threshold") else ln) for ln in cfg]
    (tmp_path / "config").write_text("\n".join(cfg) + "\n")
    cwd = os.getcwd()
    os.chdir(str(tmp_path))
    try:
        assert G.run_config("config") == []
    finally:
        os.chdir(cwd)
    r = subprocess.run([G.DRIVER_PATH, "config"], cwd=str(tmp_path), capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    assert (tmp_path / "picks.lst").read_text() == ""


def test_status_codes_keep_context_usable():
    ds = synth.make_dataset(3, nx=400, ny=352, n_templates=2, tsize=56, n_particles=1, snr=0.3,
                            n_blobs=20, ball_radius=16.0, phistep=90.0, diameter=48.0, window=128,
                            overlap=32)
    m = ds.micrographs[0]
    ctf = (m.defocus, m.dfdiff, m.dfang)
    gp = G.default_params(apix=1.0, phi_step=90.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0,
                          lowres=100.0, d_m=48.0, thres=0.0, window_size=128, overlap=32, phase_flip=1)
    with G.Context(0) as ctx:
        with pytest.raises(G.GisspaError) as e:           # search before templates
            ctx.search(m.image, ctf)
        assert e.value.status == 4
        bad = G.default_params(apix=1.0, phi_step=90.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0,
                               lowres=100.0, d_m=-1.0, thres=0.0, window_size=128, overlap=32)
        with pytest.raises(G.GisspaError) as e:           # d_m missing
            ctx.set_templates(bad, ds.templates, ctf)
        assert e.value.status == 1
        ctx.set_templates(gp, ds.templates, ctf)
        over = G.default_params(apix=1.0, phi_step=90.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0,
                                lowres=100.0, d_m=48.0, thres=0.0, window_size=128, overlap=200,
                                phase_flip=1)
        ctx2 = G.Context(0)
        ctx2.set_templates(over, ds.templates, ctf)
        with pytest.raises(G.GisspaError) as e:           # overlap >= window
            ctx2.search(m.image, ctf)
        assert e.value.status == 1
        ctx2.close()
        a = ctx.search(m.image, ctf)                       # the first context still works
        b = ctx.search(m.image, ctf)
        assert np.array_equal(a, b)
