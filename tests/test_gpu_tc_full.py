"""All-tensor-core correlation (tccorr2.cuh: every DFT stage of both passes
as FP16 tcgen05 GEMMs, FP32 accumulation, window 720) against the FP64
oracle and the FP32 CUDA path.

Tolerances: scores within 1e-3 relative of the oracle (the bound stated for
the tensor-core path; the observed error is printed); a peak may move only
between near-equal pixels (at most 1 % of the units, each keeping its score
within the bound); picks identical except lines whose score lies within 1e-3
of the threshold."""
import numpy as np
import pytest

import gisspa_b200 as G
from gisspa_b200 import synth
from oracle import gisspa_oracle as O

pytestmark = pytest.mark.gpu

TC_RTOL = 1e-3
MODES = {"tc_full": G.GS_PREC_TC_FULL, "tc_full_1p": G.GS_PREC_TC_FULL_1P}


def _case(seed, nt=6, phase_flip=1, astig=300.0):
    l, overlap = 720, 200
    return synth.make_dataset(seed, nx=int(l * 1.9), ny=int(l * 1.3), n_templates=nt, tsize=110,
                              n_particles=3, snr=0.3, n_blobs=60, ball_radius=35.0, phistep=120.0,
                              diameter=100.0, window=l, overlap=overlap, defocus=(1.0, 2.0), astig_A=astig)


@pytest.mark.parametrize("mode", sorted(MODES))
@pytest.mark.parametrize("phase_flip", [1, 0])
def test_tc_full_matches_oracle(mode, phase_flip):
    l, overlap = 720, 200
    ds = _case(31 + phase_flip, phase_flip=phase_flip)
    m = ds.micrographs[0]
    ctf = (m.defocus, m.dfdiff, m.dfang)
    p = O.Params(apix=1.0, phi_step=120.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=100.0,
                 d_m=100.0, thres=0.0, padding_size=l, phase_flip=phase_flip, overlap=overlap)
    ref = O.search(m.image, ds.templates, p, O.make_ctf(p, *ctf, l), workers=4)
    out = {}
    for prec in (G.GS_PREC_FP32, MODES[mode]):
        gp = G.default_params(apix=1.0, phi_step=120.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0,
                              lowres=100.0, d_m=100.0, thres=0.0, window_size=l, overlap=overlap,
                              phase_flip=phase_flip, precision=prec)
        with G.Context(0) as ctx:
            ctx.set_templates(gp, ds.templates, ctf)
            ctx.search(m.image, ctf)
            out[prec] = ctx.units(ref.score.shape)
    u = out[MODES[mode]]
    fin = np.isfinite(ref.score)
    assert np.array_equal(fin, np.isfinite(u["score"]))
    rel = np.abs(u["score"][fin] - ref.score[fin]) / np.abs(ref.score[fin])
    moved = (u["pos"] != ref.pos) & fin
    print("%s phase_flip %d l=720: max rel score error vs FP64 %.3e (median %.2e) over %d units, "
          "%d peaks moved" % (mode, phase_flip, rel.max(), np.median(rel), fin.sum(), moved.sum()))
    assert rel.max() <= TC_RTOL, rel.max()
    assert moved.sum() <= max(2, fin.sum() // 100), moved.sum()
    # sigma and peak come back unscaled: same as the FP32 path within the bound
    f32 = out[G.GS_PREC_FP32]
    rs = np.abs(u["sigma"][fin] - f32["sigma"][fin]) / np.abs(f32["sigma"][fin])
    assert rs.max() <= TC_RTOL, rs.max()
    same = fin & ~moved
    rp = np.abs(u["peak"][same] - f32["peak"][same]) / np.maximum(np.abs(f32["peak"][same]), 1e-30)
    assert rp.max() <= TC_RTOL, rp.max()


@pytest.mark.parametrize("mode", sorted(MODES))
def test_tc_full_picks_match_fp32(mode):
    """Threshold picks of the all-tensor-core path equal the FP32 path's,
    except lines whose score lies within 1e-3 of the threshold."""
    l, overlap = 720, 200
    ds = _case(41, nt=10)
    m = ds.micrographs[0]
    ctf = (m.defocus, m.dfdiff, m.dfang)
    picks = {}
    for prec in (G.GS_PREC_FP32, MODES[mode]):
        gp = G.default_params(apix=1.0, phi_step=120.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0,
                              lowres=100.0, d_m=100.0, thres=4.0, window_size=l, overlap=overlap,
                              phase_flip=1, precision=prec)
        with G.Context(0) as ctx:
            ctx.set_templates(gp, ds.templates, ctf)
            picks[prec] = ctx.search(m.image, ctf)
    key = lambda q: (int(q["angle_index"]), int(q["window_x"]), int(q["window_y"]), int(q["template_index"]))
    a = {key(q): q for q in picks[G.GS_PREC_FP32]}
    b = {key(q): q for q in picks[MODES[mode]]}
    assert len(a) > 0
    for k in set(a) ^ set(b):
        q = a.get(k, b.get(k))
        assert abs(float(q["score"]) - 4.0) <= TC_RTOL * 4.0, q
    for k in set(a) & set(b):
        assert abs(float(a[k]["score"]) - float(b[k]["score"])) <= TC_RTOL * abs(float(a[k]["score"]))


def test_tc_full_refuses_other_windows():
    ds = synth.make_dataset(3, nx=1000, ny=700, n_templates=2, tsize=110, n_particles=1, snr=0.3,
                            n_blobs=20, ball_radius=30.0, phistep=120.0, diameter=100.0, window=512,
                            overlap=100)
    m = ds.micrographs[0]
    gp = G.default_params(apix=1.0, phi_step=120.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0,
                          lowres=100.0, d_m=100.0, thres=0.0, window_size=512, overlap=100,
                          phase_flip=1, precision=G.GS_PREC_TC_FULL)
    with G.Context(0) as ctx:
        ctx.set_templates(gp, ds.templates, (m.defocus, m.dfdiff, m.dfang))
        with pytest.raises(G.GisspaError) as e:
            ctx.search(m.image, (m.defocus, m.dfdiff, m.dfang))
        assert e.value.status == G.GS_ERR_UNSUPPORTED
