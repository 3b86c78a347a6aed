"""Persistent correlation launches covering several in-plane angles
(GS_OPT_ANGLES_PER_LAUNCH): the dense (angle, window, template) table must be
the same whatever the grouping -- one angle per launch, a count that does not
divide the angle count, all angles in one launch, the library's own choice,
the autotuner's choice and the CUDA-graph angle loop -- with identical peak
positions and scores within 1e-6 relative (only the order of the
floating-point sum-of-squares atomics may differ).  Covers the FP32 kernel
(window 512) and the all-tensor-core kernel (window 720), whose pair spectra,
FP16 copies and per-pair maxima are laid out angle after angle."""
import numpy as np
import pytest

import gisspa_b200 as G
from gisspa_b200 import synth

pytestmark = pytest.mark.gpu

PHISTEP = 30.0          # 12 angles


@pytest.fixture(scope="module", autouse=True)
def _built():
    from gisspa_b200 import build
    build.build_library()


def _data(window, overlap, nx, ny, seed):
    ds = synth.make_dataset(seed, nx=nx, ny=ny, n_templates=7, tsize=110, n_particles=4,
                            snr=0.3, n_blobs=60, ball_radius=35.0, phistep=PHISTEP,
                            diameter=100.0, window=window, overlap=overlap, defocus=(1.0, 2.0),
                            astig_A=300.0)
    m = ds.micrographs[0]
    return ds.templates, m.image, (m.defocus, m.dfdiff, m.dfang)


def _params(window, overlap, precision):
    return G.default_params(apix=1.0, phi_step=PHISTEP, kk=3.0, energy=300.0, cs=2.7, highres=8.0,
                            lowres=100.0, d_m=100.0, thres=2.0, window_size=window, overlap=overlap,
                            phase_flip=1, precision=precision)


def _run(tmpl, img, ctf, window, overlap, precision, angles=None, graph=False, autotune=False):
    with G.Context(0) as ctx:
        if angles is not None:
            ctx.set_angles_per_launch(angles)
        if graph:
            ctx.set_graph(True)
        if autotune:
            ctx.set_autotune(True)
        ctx.set_templates(_params(window, overlap, precision), tmpl, ctf)
        picks = ctx.search(img, ctf)
        units = ctx.units()
        return units, picks, ctx.angles_per_launch()


def _same_units(a, b, rtol=1e-6):
    assert a.shape == b.shape
    assert np.array_equal(a["pos"], b["pos"])
    for f in ("score", "peak", "sigma"):
        den = np.maximum(np.abs(b[f]), 1e-30)
        rel = np.abs(a[f] - b[f]) / den
        assert rel.max() <= rtol, (f, rel.max())


def _same_picks(a, b, rtol=1e-6):
    assert len(a) == len(b)
    for f in ("angle_index", "window_x", "window_y", "template_index", "center_x", "center_y"):
        assert np.array_equal(a[f], b[f]), f
    if len(a):
        assert (np.abs(a["score"] - b["score"]) / np.abs(b["score"])).max() <= rtol


CASES = [
    # (window, overlap, nx, ny, precision)
    (512, 120, 1100, 1024, G.GS_PREC_FP32),
    (720, 200, 1240, 1240, G.GS_PREC_TC_FULL_1P),
]


@pytest.mark.parametrize("window,overlap,nx,ny,precision", CASES)
def test_grouped_angles_equal_single(window, overlap, nx, ny, precision):
    tmpl, img, ctf = _data(window, overlap, nx, ny, 71)
    ref_units, ref_picks, a1 = _run(tmpl, img, ctf, window, overlap, precision, angles=1)
    assert a1 == 1
    na = int(round(360.0 / PHISTEP))
    for angles, expect in ((5, 5), (na, na), (4 * na, na), (None, None)):
        units, picks, got = _run(tmpl, img, ctf, window, overlap, precision, angles=angles)
        if expect is not None:
            assert got == expect, (angles, got)
        else:
            # few units per angle here: the default puts every angle in one launch
            assert got == na, got
        _same_units(units, ref_units)
        _same_picks(picks, ref_picks)


def test_grouped_angles_graph_and_autotune():
    window, overlap = 512, 120
    tmpl, img, ctf = _data(window, overlap, 1100, 1024, 72)
    ref_units, ref_picks, _ = _run(tmpl, img, ctf, window, overlap, G.GS_PREC_FP32, angles=1)
    units, picks, got = _run(tmpl, img, ctf, window, overlap, G.GS_PREC_FP32, angles=5, graph=True)
    assert got == 5
    _same_units(units, ref_units)
    _same_picks(picks, ref_picks)
    units, picks, got = _run(tmpl, img, ctf, window, overlap, G.GS_PREC_FP32, autotune=True)
    na = int(round(360.0 / PHISTEP))
    assert got in (1, na // 4, na // 2, na), got
    print("autotuned angles per launch: %d of %d" % (got, na))
    _same_units(units, ref_units)
    _same_picks(picks, ref_picks)


def test_negative_angles_per_launch_rejected():
    with G.Context(0) as ctx:
        with pytest.raises(G.GisspaError):
            ctx.set_angles_per_launch(-1)
