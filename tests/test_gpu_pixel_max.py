"""gs_get_pixel_max: the per-pixel maximum of cc / sigma over (template,
angle) against the FP64 oracle's restatement (oracle search with
pixel_thres), on a window served by the generic FFT kernels (128) and one
served by the specialised ones (512).

Checked: every pixel that either side reports lies at or above the threshold
on the other side too (within the score tolerance of it); where both report,
values within SCORE_RTOL and the same (angle, template) except for near-ties
(at most 1 % of the pixels); and at the peak of every unit whose score
reaches the threshold, the map holds at least that score."""
import numpy as np
import pytest

import _helpers as H
import gisspa_b200 as G
from gisspa_b200 import synth
from oracle import gisspa_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("l,overlap,tsize,nx,ny,thres", [(128, 32, 56, 400, 352, 3.0),
                                                        (512, 128, 128, 1100, 900, 3.5)])
def test_pixel_max_matches_oracle(l, overlap, tsize, nx, ny, thres):
    d_m = tsize * 0.85
    ds = synth.make_dataset(11 + l, nx=nx, ny=ny, n_templates=5, tsize=tsize, n_particles=3, snr=0.3,
                            n_blobs=40, ball_radius=tsize / 3.5, phistep=90.0, diameter=d_m, window=l,
                            overlap=overlap, defocus=(1.0, 2.0), astig_A=200.0)
    m = ds.micrographs[0]
    ctf = (m.defocus, m.dfdiff, m.dfang)
    gp = G.default_params(apix=1.0, phi_step=90.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0,
                          lowres=100.0, d_m=d_m, thres=thres, window_size=l, overlap=overlap, phase_flip=1)
    with G.Context(0) as ctx:
        ctx.set_templates(gp, ds.templates, ctf)
        ctx.search(m.image, ctf)
        g = ctx.geometry(nx, ny)
        units = ctx.units((g.n_angles, g.n_windows_x * g.n_windows_y, g.n_templates))
        val, tmpl, ang = ctx.pixel_max(thres, (ny, nx))
        # a second call on the same search gives the same map
        val2, tmpl2, ang2 = ctx.pixel_max(thres, (ny, nx))
    assert np.array_equal(val, val2) and np.array_equal(tmpl, tmpl2) and np.array_equal(ang, ang2)

    p = O.Params(apix=1.0, phi_step=90.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=100.0,
                 d_m=d_m, thres=thres, padding_size=l, phase_flip=1, overlap=overlap)
    ref = O.search(m.image, ds.templates, p, O.make_ctf(p, *ctf, l), workers=4, pixel_thres=thres)
    rv, ra, rt = ref.pixel_value, ref.pixel_angle, ref.pixel_template

    got = tmpl >= 0
    have = np.isfinite(rv)
    assert got.sum() > 20, "too few pixels above the threshold for a meaningful check"
    tol = H.SCORE_RTOL * max(abs(thres), 1.0) + 1e-6
    only_got, only_ref = got & ~have, have & ~got
    assert np.all(np.abs(val[only_got] - thres) <= tol), val[only_got]
    assert np.all(np.abs(rv[only_ref] - thres) <= tol), rv[only_ref]
    both = got & have
    rel = np.abs(val[both] - rv[both]) / np.abs(rv[both])
    assert rel.max() <= H.SCORE_RTOL, rel.max()
    differ = both & ((tmpl != rt) | (ang != ra))
    assert differ.sum() <= max(2, both.sum() // 100), (differ.sum(), both.sum())
    assert np.all(val[~got] == 0.0) and np.all(ang[~got] == -1)

    # the map at each qualifying unit's peak holds at least its score
    offx = O.window_offsets(nx, l, overlap)
    offy = O.window_offsets(ny, l, overlap)
    bx = len(offx)
    sc = units["score"]
    hit = np.argwhere(np.isfinite(sc) & (sc >= thres))
    assert len(hit) > 0
    for ai, w, J in hit:
        pos = int(units["pos"][ai, w, J])
        x, y = offx[w % bx] + pos % l, offy[w // bx] + pos // l
        assert val[y, x] >= sc[ai, w, J] * (1 - 1e-6), (ai, w, J, val[y, x], sc[ai, w, J])
    print("pixel max l=%d: %d pixels, worst value error %.2e, %d index differences"
          % (l, both.sum(), rel.max(), differ.sum()))
