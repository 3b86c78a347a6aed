"""Shared small case for the refinement tests: one astigmatic micrograph,
window 128, its oracle search, the FP64 objective's inputs, and off-grid
picks built from the highest-scoring units."""
import numpy as np

from gisspa_b200 import synth
from oracle import gisspa_oracle as O
from oracle import refine_fp64 as R

L, OVERLAP, D_M = 128, 32, 48.0


def make_case(seed=7, n_templates=4):
    ds = synth.make_dataset(seed, nx=400, ny=352, n_templates=n_templates, tsize=56, n_particles=3,
                            snr=0.5, n_blobs=40, ball_radius=16.0, phistep=30.0, diameter=D_M,
                            window=L, overlap=OVERLAP, defocus=(1.2, 1.8), astig_A=400.0)
    m = ds.micrographs[0]
    p = O.Params(apix=1.0, phi_step=30.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=100.0,
                 d_m=D_M, thres=0.0, padding_size=L, phase_flip=1, overlap=OVERLAP)
    ctf = O.make_ctf(p, m.defocus, m.dfdiff, m.dfang, L)
    res = O.search(m.image, ds.templates, p, ctf, workers=4)
    img = O.preprocess_micrograph(m.image, p, ctf, workers=4)
    offx = O.window_offsets(m.image.shape[1], L, OVERLAP)
    offy = O.window_offsets(m.image.shape[0], L, OVERLAP)
    W = O.window_spectra(O.split_windows(img, offx, offy, L), p, workers=4)
    base = R.template_base(ds.templates, L)
    wc = R.weight_consts(p, L, ctf)
    parts = R.weight_parts(wc)
    mask = O.soft_mask(L, D_M)
    return dict(ds=ds, m=m, p=p, ctf=ctf, res=res, W=W, base=base, wc=wc, parts=parts, mask=mask,
                angles=O.angle_list(30.0))


def top_units(case, k):
    s = np.where(np.isfinite(case["res"].score), case["res"].score, -np.inf)
    flat = np.argsort(s, axis=None)[::-1][:k]
    return [np.unravel_index(i, s.shape) for i in flat]


def x0_of(pos):
    X, Y = pos % L, pos // L
    return ((X - L // 2) % L, (Y - L // 2) % L)
