"""Off-grid objective and adjoint gradient on the GPU (gs_score_grad,
gs_refine) against the FP64 reference (oracle/refine_fp64.py, itself checked
against finite differences on the CPU by tests/test_refine_fp64.py).

* at grid points the objective equals the search's score once the peak is
  left out of sigma as the search does (1e-4 relative);
* off the grid, score within 1e-4 and every gradient component within 2e-3
  of the FP64 gradient (relative to its magnitude, with an absolute floor of
  1e-3 of the gradient's norm); the template gradient within 2e-3 (relative
  L2);
* 20 steps of gradient ascent from the grid picks raise the score of at
  least 95 % of picks and lower none."""
import numpy as np
import pytest

import _refine_case as RC
import gisspa_b200 as G
from oracle import refine_fp64 as R

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    from gisspa_b200 import build
    build.build_library()


@pytest.fixture(scope="module")
def case():
    c = RC.make_case()
    m = c["m"]
    gp = G.default_params(apix=1.0, phi_step=30.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0,
                          lowres=100.0, d_m=RC.D_M, thres=0.0, window_size=RC.L, overlap=RC.OVERLAP,
                          phase_flip=1)
    ctx = G.Context(0)
    ctf = (m.defocus, m.dfdiff, m.dfang)
    ctx.set_templates(gp, c["ds"].templates, ctf)
    ctx.search(m.image, ctf)
    c["ctx"] = ctx
    c["units"] = ctx.units(c["res"].score.shape)
    yield c
    ctx.close()


def _picks(c, k, off_grid):
    m = c["m"]
    out = np.zeros(k, dtype=G.REFINE_PICK_DTYPE)
    for q, (ai, w, J) in enumerate(RC.top_units(c, k)):
        out[q]["window"] = w
        out[q]["template_index"] = J
        out[q]["pos"] = int(c["units"]["pos"][ai, w, J])
        out[q]["angle"] = c["angles"][ai] + (0.37 if off_grid else 0.0)
        out[q]["dx"], out[q]["dy"] = (0.13, -0.21) if off_grid else (0.0, 0.0)
        out[q]["defocus"] = m.defocus + (0.0137 if off_grid else 0.0)
        out[q]["dfdiff"] = m.dfdiff + (0.003 if off_grid else 0.0)
        out[q]["dfang"] = m.dfang + (7.0 if off_grid else 0.0)
    return out


def test_grid_objective_equals_search_score(case):
    pk = _picks(case, 12, off_grid=False)
    res = case["ctx"].score_grad(pk, with_gradient=False)
    n = float(RC.L * RC.L)
    for q, (ai, w, J) in enumerate(RC.top_units(case, 12)):
        s = float(res["score"][q])
        expect = s / np.sqrt((n - s * s) / (n - 1) - s * s / (n - 1) ** 2)
        ref = float(case["units"]["score"][ai, w, J])
        assert abs(expect - ref) / abs(ref) < 1e-4, (q, s, expect, ref)


def test_adjoint_matches_fp64_gradient(case):
    pk = _picks(case, 8, off_grid=True)
    res, tg = case["ctx"].score_grad(pk, with_gradient=True, template_gradients=True)
    worst = 0.0
    for q in range(len(pk)):
        p = pk[q]
        s, ge, gd, gth, gb = R.score_and_grad(case["base"][p["template_index"]], case["W"][p["window"]],
                                              RC.x0_of(int(p["pos"])), float(p["angle"]),
                                              (float(p["dx"]), float(p["dy"])),
                                              (float(p["defocus"]), float(p["dfdiff"]), float(p["dfang"])),
                                              case["wc"], case["parts"], case["mask"])
        assert abs(res["score"][q] - s) <= 1e-4 * abs(s), (q, res["score"][q], s)
        ref = np.array([ge, gd[0], gd[1], gth[0], gth[1], gth[2]])
        got = np.array([res[f][q] for f in ("d_angle", "d_dx", "d_dy", "d_defocus", "d_dfdiff", "d_dfang")])
        floor = 1e-3 * np.linalg.norm(ref)
        err = np.abs(got - ref) / (np.abs(ref) + floor)
        worst = max(worst, err.max())
        assert err.max() <= 2e-3, (q, got, ref)
        terr = np.linalg.norm(tg[q] - gb) / np.linalg.norm(gb)
        assert terr <= 2e-3, (q, terr)
    print("adjoint vs FP64 gradient: worst component error %.2e" % worst)


def test_autograd_function_backward(case):
    """The torch.autograd.Function wrapper: backward of sum(scores) gives the
    adjoint's gradient, which matches the FP64 reference."""
    torch = pytest.importorskip("torch")
    from gisspa_b200.autograd import PickScore, PARAM_FIELDS
    pk = _picks(case, 4, off_grid=True)
    params = torch.tensor(np.stack([pk[f].astype(np.float64) for f in PARAM_FIELDS], axis=1),
                          requires_grad=True)
    s = PickScore.apply(params, case["ctx"], pk)
    s.sum().backward()
    for q in range(len(pk)):
        p = pk[q]
        _, ge, gd, gth, _ = R.score_and_grad(case["base"][p["template_index"]], case["W"][p["window"]],
                                             RC.x0_of(int(p["pos"])), float(p["angle"]),
                                             (float(p["dx"]), float(p["dy"])),
                                             (float(p["defocus"]), float(p["dfdiff"]), float(p["dfang"])),
                                             case["wc"], case["parts"], case["mask"])
        ref = np.array([ge, gd[0], gd[1], gth[0], gth[1], gth[2]])
        got = params.grad[q].numpy()
        assert (np.abs(got - ref) <= 2e-3 * (np.abs(ref) + 1e-3 * np.linalg.norm(ref))).all(), (got, ref)


def test_refinement_improves_grid_picks(case):
    pk = _picks(case, 24, off_grid=False)
    start = case["ctx"].score_grad(pk, with_gradient=False)["score"]
    refined, res = case["ctx"].refine(pk, steps=20)
    gain = res["score"] - start
    assert (gain >= -1e-6 * np.abs(start)).all(), gain
    frac = float((gain > 1e-6 * np.abs(start)).mean())
    print("refinement: %.0f %% of picks improved, median gain %.3e" % (100 * frac, np.median(gain)))
    assert frac >= 0.95
