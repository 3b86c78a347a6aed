"""gs_search_batch (micrographs of different sizes in one search), the CUDA
graph of the angle loop and the scheduling autotuner: each must give the same
picks as plain one-micrograph searches (scores within 1e-6 relative: only the
order of floating-point accumulation may differ)."""
import numpy as np
import pytest

import gisspa_b200 as G
from gisspa_b200 import synth

pytestmark = pytest.mark.gpu

SIZES = [(1100, 1024), (900, 1150), (1230, 800)]   # (nx, ny)


@pytest.fixture(scope="module", autouse=True)
def _built():
    from gisspa_b200 import build
    build.build_library()


@pytest.fixture(scope="module")
def data():
    mics = []
    base = None
    for k, (nx, ny) in enumerate(SIZES):
        ds = synth.make_dataset(40 + k, nx=nx, ny=ny, n_templates=6, tsize=110, n_particles=4,
                                snr=0.3, n_blobs=60, ball_radius=35.0, phistep=60.0,
                                diameter=100.0, window=512, overlap=120, defocus=(1.0, 2.0),
                                astig_A=300.0)
        if base is None:
            base = ds
        m = ds.micrographs[0]
        mics.append((m.image, (m.defocus, m.dfdiff, m.dfang)))
    return base.templates, mics


def _params(precision=0):
    return G.default_params(apix=1.0, phi_step=60.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0,
                            lowres=100.0, d_m=100.0, thres=2.0, window_size=512, overlap=120,
                            phase_flip=1, precision=precision)


def _same(a, b, rtol=1e-6):
    assert len(a) == len(b), (len(a), len(b))
    for f in ("angle_index", "window_x", "window_y", "template_index", "center_x", "center_y"):
        assert np.array_equal(a[f], b[f]), f
    if len(a):
        rel = np.abs(a["score"] - b["score"]) / np.abs(b["score"])
        assert rel.max() <= rtol, rel.max()


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_equals_single_searches(data, precision):
    tmpl, mics = data
    first_ctf = mics[0][1]
    single = []
    with G.Context(0) as ctx:
        ctx.set_templates(_params(precision), tmpl, first_ctf)
        for img, ctf in mics:
            single.append(ctx.search(img, ctf))
        batch = ctx.search_batch([m[0] for m in mics], [m[1] for m in mics])
        units = ctx.units()
    assert len(batch) == len(mics)
    for a, b in zip(batch, single):
        assert len(b) > 20
        _same(a, b)
    assert units.size > 0


def test_graph_equals_stream(data):
    tmpl, mics = data
    res = []
    for graph in (False, True):
        with G.Context(0) as ctx:
            ctx.set_graph(graph)
            ctx.set_templates(_params(), tmpl, mics[0][1])
            res.append(ctx.search_batch([m[0] for m in mics], [m[1] for m in mics]))
            t = ctx.timings()
            if graph:
                assert t[1] == 0.0 and t[2] > 0.0
    for a, b in zip(*res):
        _same(a, b)


def test_autotuned_equals_default(data):
    tmpl, mics = data
    img, ctf = mics[0]
    with G.Context(0) as ctx:
        ctx.set_templates(_params(), tmpl, ctf)
        ref = ctx.search(img, ctf)
        # window 512, FP32: 32 ring slots, lag 10, window block 8, 8-vector tiles
        assert ctx.tuning() == (32, 10, 8, 0, 8)
    with G.Context(0) as ctx:
        ctx.set_autotune(True)
        ctx.set_templates(_params(), tmpl, ctf)
        got = ctx.search(img, ctf)
        slots, lag, wb, ctas, tile = ctx.tuning()
        again = ctx.search(img, ctf)          # cached choice
        assert ctx.tuning() == (slots, lag, wb, ctas, tile)
    print("autotuned scheduling: slots %d lag %d window block %d ctas/SM %d tile %d"
          % (slots, lag, wb, ctas, tile))
    assert 0 <= lag < slots and wb >= 1 and ctas >= 0 and tile in (8, 16)
    _same(got, ref)
    _same(again, ref)


def test_narrow_tiles_equal_wide(data):
    """The persistent kernel with 8-vector tiles (four 128-thread CTAs per
    SM) against the default 16-vector tiles."""
    tmpl, mics = data
    res = []
    for tile in (16, 8):
        with G.Context(0) as ctx:
            ctx.set_corr_tile(tile)
            ctx.set_templates(_params(), tmpl, mics[0][1])
            res.append(ctx.search_batch([m[0] for m in mics], [m[1] for m in mics]))
            assert ctx.tuning()[4] == tile
    for a, b in zip(*res):
        _same(a, b)


def test_two_pass_batch(data):
    tmpl, mics = data
    res = []
    for two_pass in (False, True):
        with G.Context(0) as ctx:
            ctx.set_two_pass(two_pass)
            ctx.set_templates(_params(), tmpl, mics[0][1])
            res.append(ctx.search_batch([m[0] for m in mics], [m[1] for m in mics]))
    for a, b in zip(*res):
        _same(a, b)
