"""The C++/OpenMP CPU baseline (oracle/cpu/gisspa_cpu.cpp) against the FP64
oracle: every (window, template) unit of one in-plane angle, on a window of
the generic sizes (128) and the full-size one (720).  It is the CPU arm bench.py
times, so it must compute the same scores (within the FP32 tolerance) and
peak positions.  No GPU."""
import ctypes

import numpy as np
import pytest

import _helpers as H
from gisspa_b200 import build, synth
from oracle import gisspa_oracle as O


@pytest.mark.parametrize("l,overlap,tsize,nx,ny", [(128, 32, 56, 400, 352), (720, 200, 110, 1500, 800)])
def test_cpu_baseline_matches_oracle(l, overlap, tsize, nx, ny):
    lib = ctypes.CDLL(build.build_cpu_baseline())
    d_m = tsize * 0.85
    ds = synth.make_dataset(3 + l, nx=nx, ny=ny, n_templates=5, tsize=tsize, n_particles=3, snr=0.3,
                            n_blobs=40, ball_radius=tsize / 3.5, phistep=90.0, diameter=d_m, window=l,
                            overlap=overlap, defocus=(1.0, 2.0), astig_A=200.0)
    m = ds.micrographs[0]
    ctf = (m.defocus, m.dfdiff, m.dfang)
    p = O.Params(apix=1.0, phi_step=90.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=100.0,
                 d_m=d_m, thres=3.0, padding_size=l, phase_flip=1, overlap=overlap)
    oc = O.make_ctf(p, *ctf, l)
    ai = 1
    ref = O.search(m.image, ds.templates, p, oc, workers=4, angles=[ai])
    T = O.prepare_templates(ds.templates, p, l, oc, workers=4)
    img = O.preprocess_micrograph(m.image, p, oc, workers=4)
    W = O.window_spectra(O.split_windows(img, O.window_offsets(nx, l, overlap), O.window_offsets(ny, l, overlap),
                                         l), p, workers=4).astype(np.complex64)
    TS = O.template_spectra(T, O.angle_list(90.0)[ai], d_m, workers=4).astype(np.complex64)
    nw, nt = W.shape[0], TS.shape[0]
    sc = np.zeros(nw * nt, np.float32)
    pos = np.zeros(nw * nt, np.int32)
    r = lib.gsc_correlate(ctypes.c_void_p(W.ctypes.data), nw, ctypes.c_void_p(TS.ctypes.data), nt, l,
                          ctypes.c_float(d_m), ctypes.c_void_p(sc.ctypes.data), ctypes.c_void_p(pos.ctypes.data), 2)
    assert r == 0
    rs, rp = ref.score[ai].ravel(), ref.pos[ai].ravel()
    fin = np.isfinite(rs)
    assert np.array_equal(fin, np.isfinite(sc))
    rel = np.abs(sc[fin] - rs[fin]) / np.abs(rs[fin])
    assert rel.max() <= H.SCORE_RTOL, rel.max()
    assert np.array_equal(pos[fin], rp[fin])


def test_cpu_baseline_rejects_other_sizes():
    lib = ctypes.CDLL(build.build_cpu_baseline())
    buf = np.zeros(2 * 7 * 7, np.float32)
    out = np.zeros(4, np.float32)
    assert lib.gsc_correlate(ctypes.c_void_p(buf.ctypes.data), 1, ctypes.c_void_p(buf.ctypes.data), 1, 7,
                             ctypes.c_float(2.0), ctypes.c_void_p(out.ctypes.data),
                             ctypes.c_void_p(out.ctypes.data), 1) == -1
