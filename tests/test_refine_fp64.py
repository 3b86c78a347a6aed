"""The FP64 refinement objective (oracle/refine_fp64.py) itself, on the CPU:
at the grid point it reproduces the search's score, its template base
rebuilds the search's preprocessed templates, and its autograd gradient
agrees with central finite differences (step 1e-3) at off-grid points."""
import numpy as np
import torch

import _refine_case as RC
from oracle import gisspa_oracle as O
from oracle import refine_fp64 as R


def test_base_and_grid_score():
    c = RC.make_case()
    T = O.prepare_templates(c["ds"].templates, c["p"], RC.L, c["ctf"])
    m = c["m"]
    theta = (m.defocus, m.dfdiff, m.dfang)
    for J in range(T.shape[0]):
        bt = torch.tensor(c["base"][J])
        F1 = torch.fft.fft2(bt) / RC.L ** 2 * R.weight_torch(c["wc"], torch.tensor(theta, dtype=torch.float64), c["parts"])
        y, x = np.mgrid[0:RC.L, 0:RC.L]
        sel = torch.as_tensor((x <= RC.L // 2) & c["parts"][1])
        a = torch.sqrt((F1.real ** 2 + F1.imag ** 2)[sel].sum()) / float(sel.sum())
        t = (torch.fft.ifft2(F1 / a).real * RC.L ** 2).numpy()
        # the oracle rounds dfu, dfv to float32 (astigmatic case): 1e-6 relative
        assert np.abs(t - T[J]).max() <= 1e-6 * np.abs(T[J]).max()
    for (ai, w, J) in RC.top_units(c, 5):
        pos = int(c["res"].pos[ai, w, J])
        s, *_ = R.score_and_grad(c["base"][J], c["W"][w], RC.x0_of(pos), float(c["angles"][ai]), (0.0, 0.0),
                                 theta, c["wc"], c["parts"], c["mask"])
        ref = c["res"].score[ai, w, J]
        # the search's sigma leaves the peak out (main.cu:869-876): with the
        # map's zero mean, sigma_ref^2 = (n sig^2 - peak^2) / (n - 1) -
        # (peak / (n - 1))^2, n = l^2, so score_ref follows from s exactly
        n = float(RC.L * RC.L)
        expect = s / np.sqrt((n - s * s) / (n - 1) - s * s / (n - 1) ** 2)
        assert abs(expect - ref) / abs(ref) < 1e-4, (s, expect, ref)


def test_autograd_matches_finite_differences():
    c = RC.make_case()
    m = c["m"]
    # a generic point: away from |CTF| zero crossings, where the objective has kinks
    theta0 = np.array([m.defocus + 0.0137, m.dfdiff + 0.003, m.dfang + 7.0])
    (ai, w, J) = RC.top_units(c, 1)[0]
    pos = int(c["res"].pos[ai, w, J])
    x0 = RC.x0_of(pos)
    e0, d0 = float(c["angles"][ai]) + 0.37, np.array([0.13, -0.21])
    s, ge, gd, gth, gb = R.score_and_grad(c["base"][J], c["W"][w], x0, e0, d0, theta0, c["wc"],
                                          c["parts"], c["mask"])

    def f(e=e0, d=d0, th=theta0, b=None):
        bb = c["base"][J] if b is None else b
        return float(R.score_torch(torch.tensor(bb), torch.tensor(c["W"][w]), x0,
                                   torch.tensor(float(e), dtype=torch.float64),
                                   torch.tensor(np.asarray(d, dtype=np.float64)),
                                   torch.tensor(np.asarray(th, dtype=np.float64)),
                                   c["wc"], c["parts"], c["mask"]))
    h = 1e-3
    # the bilinear rotation has kinks where a source coordinate crosses a
    # pixel edge (about 0.2 % of them move across one in +-1e-3 deg): 1e-5 deg
    he = 1e-5
    fd = [(f(e=e0 + he) - f(e=e0 - he)) / (2 * he)]
    for k in range(2):
        dp, dm = d0.copy(), d0.copy()
        dp[k] += h
        dm[k] -= h
        fd.append((f(d=dp) - f(d=dm)) / (2 * h))
    # |CTF| has kinks at its zeros; a step of 1e-3 um moves about 0.6 % of
    # the in-band zeros across some pixel, so the two defocus magnitudes use
    # 1e-5 um (dfang, in degrees, keeps 1e-3)
    for k, hk in zip(range(3), (1e-5, 1e-5, h)):
        tp, tm = theta0.copy(), theta0.copy()
        tp[k] += hk
        tm[k] -= hk
        fd.append((f(th=tp) - f(th=tm)) / (2 * hk))
    ag = [ge, gd[0], gd[1], gth[0], gth[1], gth[2]]
    for a_, f_ in zip(ag, fd):
        assert abs(a_ - f_) <= 1e-3 * abs(f_) + 1e-5, (ag, fd)
    # template pixels: a few of the largest-gradient pixels
    idx = np.argsort(np.abs(gb).ravel())[::-1][:3]
    for i in idx:
        bp, bm = c["base"][J].copy(), c["base"][J].copy()
        scale = max(1.0, np.abs(c["base"][J]).max()) * 1e-6
        bp.ravel()[i] += scale
        bm.ravel()[i] -= scale
        fdv = (f(b=bp) - f(b=bm)) / (2 * scale)
        assert abs(gb.ravel()[i] - fdv) <= 1e-3 * abs(fdv) + 1e-12, (gb.ravel()[i], fdv)
