"""gs_correlate_window_noalloc: the correlation of one window with all
templates, for callers that may not allocate device memory while they run
(for example code being captured into a CUDA graph).  Its intermediate maps
live in the library's fixed static scratch array, so the call itself never
allocates; the caller owns the input and output buffers (allocated here with
torch, outside the call).

The check: its per-template results for one (angle, window) must equal those
the full search (gs_search, the existing entry point) reports for the same
unit, within the score tolerance used throughout the tests, on two calls in a
row (the second call reuses the scratch the first one left behind).  This
file is collected last so that a failure here cannot hide other results."""
import numpy as np
import pytest

import _helpers as H
import gisspa_b200 as G
from gisspa_b200 import synth
from oracle import gisspa_oracle as O

pytestmark = pytest.mark.gpu


def _case(l, overlap, tsize, nt, seed):
    nx, ny = max(int(l * 1.9), 400), max(int(l * 1.3), 352)
    ds = synth.make_dataset(seed, nx=nx, ny=ny, n_templates=nt, tsize=tsize,
                            n_particles=2, snr=0.3, n_blobs=40, ball_radius=tsize / 3.5,
                            phistep=90.0, diameter=tsize * 0.9, window=l, overlap=overlap,
                            defocus=(1.0, 2.0), astig_A=250.0)
    return ds


@pytest.mark.parametrize("l,overlap,tsize,nt", [(720, 200, 110, 3), (128, 32, 56, 5)])
def test_noalloc_matches_search(l, overlap, tsize, nt):
    torch = pytest.importorskip("torch")
    from gisspa_b200 import build
    build.build_library()
    ds = _case(l, overlap, tsize, nt, seed=31 + l)
    m = ds.micrographs[0]
    d_m = float(ds.params["diameter"])
    gp = G.default_params(apix=1.0, phi_step=90.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0,
                          lowres=100.0, d_m=d_m, thres=0.0, window_size=l, overlap=overlap,
                          phase_flip=1)
    ctf = (m.defocus, m.dfdiff, m.dfang)
    with G.Context(0) as ctx:
        ctx.set_templates(gp, ds.templates, ctf)
        ctx.search(m.image, ctf)
        g = ctx.geometry(m.image.shape[1], m.image.shape[0])
        nw = g.n_windows_x * g.n_windows_y
        units = ctx.units((g.n_angles, nw, nt))

    # the same window and template-pair spectra, built on the host by the oracle
    p = O.Params(apix=1.0, phi_step=90.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=100.0,
                 d_m=d_m, thres=0.0, padding_size=l, phase_flip=1, overlap=overlap)
    oc = O.make_ctf(p, *ctf, l)
    T = O.prepare_templates(ds.templates, p, l, oc, workers=4)
    img = O.preprocess_micrograph(m.image, p, oc, workers=4)
    offx = O.window_offsets(m.image.shape[1], l, overlap)
    offy = O.window_offsets(m.image.shape[0], l, overlap)
    W = O.window_spectra(O.split_windows(img, offx, offy, l), p, workers=4)
    ai = 1
    TS = O.template_spectra(T, O.angle_list(90.0)[ai], d_m, workers=4)
    npairs = (nt + 1) // 2
    P = np.zeros((npairs, l, l), dtype=np.complex128)
    for q in range(npairs):
        P[q] = TS[2 * q] - (1j * TS[2 * q + 1] if 2 * q + 1 < nt else 0.0)

    dev = torch.device("cuda", 0)
    d_P = torch.from_numpy(P.astype(np.complex64)).to(dev)
    d_units = torch.zeros((nt, 4), dtype=torch.float32, device=dev)
    wins = (nw - 1, 0)                               # two calls in a row, different windows
    d_Ws = [torch.from_numpy(W[w].astype(np.complex64)).to(dev) for w in wins]
    free_after_first = None
    for call, w in enumerate(wins):
        d_units.fill_(float("nan"))
        torch.cuda.synchronize()
        G.correlate_window_noalloc(d_Ws[call].data_ptr(), d_P.data_ptr(), nt, l, d_m, d_units.data_ptr())
        torch.cuda.synchronize()
        # the first call may load the library's module (which holds the static
        # scratch); from then on a call takes no device memory at all
        free_now = torch.cuda.mem_get_info(dev)[0]
        if call == 0:
            free_after_first = free_now
        else:
            assert free_now == free_after_first, (free_after_first, free_now)
        got = d_units.cpu().numpy()
        score = got[:, 0]
        pos = got[:, 1].copy().view(np.int32)
        ref = units[ai, w]
        fin = np.isfinite(ref["score"])
        assert np.array_equal(fin, np.isfinite(score)), (call, w)
        rel = np.abs(score[fin] - ref["score"][fin]) / np.abs(ref["score"][fin])
        assert rel.max() <= H.SCORE_RTOL, (call, w, rel.max())
        assert np.array_equal(pos[fin], ref["pos"][fin]), (call, w)


def test_noalloc_rejects_oversized_window():
    torch = pytest.importorskip("torch")
    big = G.NOALLOC_MAX_WINDOW + 2
    buf = torch.zeros(8, dtype=torch.float32, device="cuda")
    with pytest.raises(G.GisspaError) as e:
        G.correlate_window_noalloc(buf.data_ptr(), buf.data_ptr(), 2, big, 50.0, buf.data_ptr())
    assert e.value.status == 5  # GS_ERR_UNSUPPORTED
    with pytest.raises(G.GisspaError) as e:
        G.correlate_window_noalloc(buf.data_ptr(), buf.data_ptr(), 2, 101, 50.0, buf.data_ptr())
    assert e.value.status == 1  # odd window: GS_ERR_ARG
