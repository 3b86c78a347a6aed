"""FP64 CPU restatement of the GisSPA 2D template-matching search (norm_type 0).

TEST INFRASTRUCTURE ONLY.  This module is the parity checker for the CUDA
path in ``gisspa_b200``: tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may call it; the product never does.

It restates, step by step, what the reference computes (file:line cited on
every function, paths relative to the GisSPA repository), in float64 NumPy /
SciPy (pocketfft) arithmetic.  Wherever the reference takes a *discrete*
decision from float32 arithmetic, the float32 arithmetic is emulated so that
the decision is the same:

* hot-pixel bounds from sequential float32 sums (main.cu:529-543);
* the in-plane angle loop accumulated in float32 (main.cu:1232);
* cos/sin of the angle rounded to float32 (GPU_func.cu:498-499);
* radial shell indices from float32 ``hypotf`` (GPU_func.cu:119, 138, 167);
* band-pass limits such as ``l*apix/highres`` formed in float32.

Everything continuous (FFTs, whitening, CTF weighting, interpolation,
correlation, sigma) is float64, so the oracle sits at the FP64 answer and
the reference's own float32 noise is what a parity tolerance must absorb.

Parity pin: ``tests/golden/`` holds outputs of the reference itself (built
from its own sources by ``oracle/Makefile`` and run on a B200), and
``tests/test_oracle_golden.py`` checks this module against them.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace
from typing import List, Optional, Sequence, Tuple

import numpy as np
import scipy.fft as sfft

PI_REF = 3.141592654  # GPU_func.cuh:29 (double literal used by every kernel)
EPS_REF = 1e-8        # GPU_func.cuh:28
RA_SIZE = 5000        # GPU_func.cuh:31 (radial-shell buffer per image)

f32 = np.float32


# ---------------------------------------------------------------------------
# Parameters (DataReader.h:14-42) and per-micrograph CTF state (main.cu:140-156)
# ---------------------------------------------------------------------------
@dataclass
class Params:
    """Mirror of the reference ``struct Parameters`` (EMReader/DataReader.h:14-42).

    Scalars are kept as Python floats but every use goes through float32, as
    in the reference."""

    apix: float = -1.0
    phi_step: float = -1.0
    kk: float = -1.0
    energy: float = -1.0
    cs: float = -1.0
    highres: float = -1.0
    lowres: float = -1.0
    d_m: float = -1.0
    edge_half_width: float = 6.0
    ampconst: float = 0.07
    a: float = -9.32
    b: float = 2.65
    b2: float = 0.01908
    bfactor: float = -78.7757
    bfactor2: float = -12.9121
    bfactor3: float = 1.28732
    first: int = -1
    last: int = -1
    thres: float = 7.0
    padding_size: int = 320
    phase_flip: int = 0
    overlap: int = -1
    invert: int = 0
    norm_type: int = 0


@dataclass
class Ctf:
    """Per-micrograph CTF state as ``readRawImage`` leaves it (main.cu:150-155)."""

    defocus: float  # negated on parse (DataReader.cpp:377)
    dfdiff: float
    dfang: float
    dfu: float
    dfv: float
    lam: float
    ds: float


def make_ctf(p: Params, defocus_um: float, dfdiff_um: float, dfang_deg: float,
             padding_size: int) -> Ctf:
    """main.cu:150-155 and DataReader.cpp:375-385, with float32 storage."""
    defocus = f32(-f32(defocus_um))
    dfdiff = f32(dfdiff_um)
    dfang = f32(dfang_deg)
    dfu = f32(defocus + dfdiff)
    dfv = f32(defocus - dfdiff)
    e = float(f32(p.energy))
    lam = f32(12.2639 / math.sqrt(e * 1000.0 + 0.97845 * e * e))
    ds = f32(f32(1.0) / f32(f32(p.apix) * f32(padding_size)))
    return Ctf(float(defocus), float(dfdiff), float(dfang), float(dfu), float(dfv),
               float(lam), float(ds))


# ---------------------------------------------------------------------------
# Small shared pieces
# ---------------------------------------------------------------------------
def hypotf_int(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """float32 ``hypotf`` of integer arguments (correctly rounded)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.sqrt(a * a + b * b).astype(np.float32)


def shell_index(nx: int, ny: int) -> np.ndarray:
    """``floor(hypotf(min(y,ny-y), min(x,nx-x)) + 0.5) - 1`` (GPU_func.cu:119,138,167)."""
    y, x = np.mgrid[0:ny, 0:nx]
    h = hypotf_int(np.minimum(y, ny - y), np.minimum(x, nx - x))
    return (np.floor(h.astype(np.float64) + 0.5) - 1).astype(np.int64)


def ctf_ast(x1: np.ndarray, y1: np.ndarray, nx: int, ny: int, apix: float,
            dfu: float, dfv: float, dfdiff: float, dfang: float, lam: float,
            cs: float, ampconst: float, mode: int) -> np.ndarray:
    """Astigmatic CTF, GPU_func.cu:292-315.  mode 0 = sign, 2 = |CTF|, else value.

    ``x1`` / ``y1`` are the integer indices the call sites pass
    (x, (y + ny/2) % ny)."""
    x1 = np.asarray(x1, dtype=np.int64)
    y1 = np.asarray(y1, dtype=np.int64)
    y1 = np.where(x1 > nx // 2, ny - y1, y1)
    x1 = np.minimum(x1, nx - x1)
    dx = x1.astype(np.float64)
    dy = (y1 - ny // 2).astype(np.float64)
    apix = float(f32(apix))
    ss = (dx * dx / float(nx * nx) + dy * dy / float(ny * ny)) / (apix * apix)
    ag = np.arctan2(dy, dx)
    df_ast = 0.5 * (dfu + dfv + 2.0 * dfdiff * np.cos(2.0 * (dfang * PI_REF / 180.0 - ag)))
    gamma = -2.0 * PI_REF * (cs * 2.5e6 * lam ** 3 * ss * ss + df_ast * 5000.0 * lam * ss)
    a = float(f32(ampconst))
    v = math.sqrt(1.0 - a * a) * np.sin(gamma) + a * np.cos(gamma)
    if mode == 0:
        return np.where(v > 0, 1.0, -1.0)
    if mode == 2:
        return np.abs(v)
    return v


def _bandpass(r: np.ndarray, hp: float, lp: float, low_cut: bool) -> np.ndarray:
    """Band-pass factor on shell index ``r`` with 8-px cosine edges.

    Template form (GPU_func.cu:270-278, ``low_cut=False``): the pass branch
    accepts every 0 <= r < hp, so no low cut is applied.  Micrograph form
    (GPU_func.cu:183-191, ``low_cut=True``): pass only for lp <= r < hp."""
    r = r.astype(np.float64)
    out = np.zeros_like(r)
    if low_cut:
        pas = (r < hp) & (r >= lp)
    else:
        pas = (r < hp) & (r >= 0)
    hi = (~pas) & (r >= hp) & (r < hp + 8)
    lo = (~pas) & (~hi) & (r >= lp - 8) & (r < lp) & (r >= 0)
    out[pas] = 1.0
    out[hi] = 0.5 * np.cos(PI_REF * (r[hi] - hp) / 16.0) + 0.5
    out[lo] = 0.5 * np.cos(PI_REF * (lp - r[lo]) / 16.0) + 0.5
    return out


def _fft2(a, workers):
    return sfft.fft2(a, axes=(-2, -1), workers=workers)


def _ifft2_unnorm(a, workers):
    """cuFFT's unnormalised inverse (exp(+2 pi i ...), no 1/n)."""
    return sfft.ifft2(a, axes=(-2, -1), norm="forward", workers=workers)


# ---------------------------------------------------------------------------
# Geometry
# ---------------------------------------------------------------------------
def adjust_padding_size(window_size: int, tx: int, ty: int) -> int:
    """main.cu:158-178: smallest multiple of 32 >= the template, only if the
    configured window is smaller than the template."""
    if window_size < tx or window_size < ty:
        l = 0
        while l < tx or l < ty:
            l += 32
        return l
    return window_size


def window_offsets(n: int, l: int, overlap: int) -> List[int]:
    """Window origins along one axis, last one snapped to n - l (main.cu:228-250)."""
    interval = l - overlap
    if interval <= 0:
        raise ValueError("overlap must be smaller than the window size")
    offs = [0]
    off = 0
    while off + l < n:
        off += interval
        if off + l >= n:
            off = n - l
        offs.append(off)
    return offs


def angle_list(phi_step: float) -> List[np.float32]:
    """In-plane angles of the search loop, accumulated in float32 (main.cu:1232)."""
    step = f32(phi_step)
    if not step > 0:
        raise ValueError("phistep must be positive")
    out = []
    e = f32(0.0)
    while e < f32(360.0):
        out.append(e)
        e = f32(e + step)
    return out


def printed_phi(euler3: np.float32) -> np.float32:
    """Third Euler angle written to the .lst: 360 - euler3 wrapped (main.cu:1254-1256)."""
    cur = f32(f32(360.0) - f32(euler3))
    if cur >= f32(360.0):
        cur = f32(cur - f32(360.0))
    return cur


# ---------------------------------------------------------------------------
# Templates (once per run): main.cu:182-474
# ---------------------------------------------------------------------------
def pad_templates(raw: np.ndarray, l: int) -> np.ndarray:
    """Centre-pad each t_y x t_x template into l x l (main.cu:182-223)."""
    n, ty, tx = raw.shape
    out = np.zeros((n, l, l), dtype=np.float64)
    sx = (l - tx) // 2
    sy = (l - ty) // 2
    out[:, sy:sy + ty, sx:sx + tx] = raw.astype(np.float32)
    return out


def edge_normalize(T: np.ndarray) -> np.ndarray:
    """(t - ring mean) / sigma over the whole frame (main.cu:311-385, K1-K4).

    The ring is the 1-px annulus (r-1)^2 <= d^2 <= (r+1)^2, r = l/2 - 2,
    around (l/2, l/2); sigma is the std of the full padded l x l frame."""
    n, l, _ = T.shape
    r = f32(f32(l) / f32(2) - f32(2))
    up = low = f32(0)
    if r > 1:
        up = f32((r + 1) * (r + 1))
        low = f32((r - 1) * (r - 1))
    y, x = np.mgrid[0:l, 0:l]
    rr = ((x - l // 2) ** 2 + (y - l // 2) ** 2).astype(np.float32)
    ring = (rr >= low) & (rr <= up)
    count = ring.sum()
    em = T[:, ring].sum(axis=1) / count
    mean = T.reshape(n, -1).mean(axis=1)
    sig2 = (T.reshape(n, -1) ** 2).mean(axis=1) - mean * mean
    with np.errstate(invalid="ignore"):
        sigma = np.sqrt(sig2)
    sigma[~np.isfinite(sigma) | (sigma < 0)] = 0.0
    out = T.copy()
    ok = np.abs(sigma) >= EPS_REF
    out[ok] = (T[ok] - em[ok, None, None]) / sigma[ok, None, None]
    return out


def template_weight_factor(p: Params, l: int, ctf0: Ctf) -> np.ndarray:
    """Per-bin band-pass x |CTF| x Wiener factor of apply_weighting_function
    (GPU_func.cu:249-290), CTF from the FIRST micrograph (main.cu:1106,1129)."""
    y, x = np.mgrid[0:l, 0:l]
    rf = hypotf_int(np.minimum(y, l - y), np.minimum(x, l - x)).astype(np.float64)
    r_round = (np.floor(rf + 0.5) - 1).astype(np.int64)
    hp = float(f32(f32(f32(l) * f32(p.apix)) / f32(p.highres)))
    lp = float(f32(f32(f32(l) * f32(p.apix)) / f32(p.lowres)))
    band = _bandpass(r_round, hp, lp, low_cut=False)
    ss = rf * float(f32(ctf0.ds))
    wsel = (r_round < l // 2) & (r_round >= 0)
    v = ctf_ast(x, (y + l // 2) % l, l, l, p.apix, ctf0.dfu, ctf0.dfv, ctf0.dfdiff,
                ctf0.dfang, ctf0.lam, float(f32(p.cs)), p.ampconst, 2)
    kk = float(f32(p.kk))
    signal = np.exp(p.bfactor * ss * ss + p.bfactor2 * ss + p.bfactor3) / (kk + 1.0)
    ncurve = np.exp(p.a * ss * ss + p.b * ss + p.b2) / signal
    w = v * np.sqrt(1.0 / (ncurve + kk * v * v))
    return band * np.where(wsel, w, 1.0)


def prepare_templates(raw: np.ndarray, p: Params, l: int, ctf0: Ctf,
                      workers: int = 1) -> np.ndarray:
    """Templates after readAndPaddingTemplate + edgeNormalize + handleTemplate
    (main.cu:182-474): real l x l images, float64, shape (N, l, l)."""
    T = edge_normalize(pad_templates(raw, l))
    n = T.shape[0]
    F = _fft2(T, workers) / float(l * l)                       # main.cu:410-412
    amp2 = (F.real ** 2 + F.imag ** 2)
    r = shell_index(l, l)
    y, x = np.mgrid[0:l, 0:l]
    half = x <= l // 2
    shell_ok = (r >= 0) & (r < l // 2)
    sel = half & shell_ok                                       # GPU_func.cu:116-121
    ridx = r[sel]
    whiten = np.ones((n, l, l))
    for k in range(n):                                          # SQRSum_by_circle + whiten_Tmp
        ra = np.bincount(ridx, weights=amp2[k][sel], minlength=l // 2)
        rb = np.bincount(ridx, minlength=l // 2).astype(np.float64)
        with np.errstate(divide="ignore", invalid="ignore"):
            fac = 1.0 / np.sqrt(ra / rb)
        wk = np.ones((l, l))
        wk[shell_ok] = fac[r[shell_ok]]
        whiten[k] = wk
    F = F * whiten * template_weight_factor(p, l, ctf0)[None]  # K6, K10
    amp2 = F.real ** 2 + F.imag ** 2                            # K12: r<l/2, x<=l/2
    s = amp2[:, sel].sum(axis=1)
    cnt = float(sel.sum())
    m = np.sqrt(s / (cnt * cnt))
    m_safe = np.where(m != 0, m, 1.0)
    F = F / m_safe[:, None, None]                               # K14
    return _ifft2_unnorm(F, workers).real                       # main.cu:463


# ---------------------------------------------------------------------------
# Per-angle template spectra: main.cu:669-716
# ---------------------------------------------------------------------------
def rotation_cos_sin(euler3: float) -> Tuple[np.float32, np.float32]:
    """``float cose = cos(e*PI/180)`` with e float, PI double (GPU_func.cu:498-499)."""
    ang = float(f32(euler3)) * PI_REF / 180.0
    return f32(math.cos(ang)), f32(math.sin(ang))


def rotate_bilinear(T: np.ndarray, euler3: float) -> np.ndarray:
    """rotate_subIMG on the real part (GPU_func.cu:496-560): output(x, y) samples
    the input at (cos e x + sin e y, -sin e x + cos e y) about (l/2, l/2)."""
    n, l, _ = T.shape
    c, s = (float(v) for v in rotation_cos_sin(euler3))
    j, i = np.mgrid[0:l, 0:l]
    x = (i - l // 2).astype(np.float64)
    y = (j - l // 2).astype(np.float64)
    # float32 source coordinates as the kernel forms them: the second product
    # rounded, the first fused into it (fma), then + l/2 rounded; the
    # out-of-frame test below is a discrete decision on these values.
    h = float(l // 2)
    x2 = (c * x + (s * y).astype(np.float32)).astype(np.float32)
    x2 = (x2 + np.float32(h)).astype(np.float32).astype(np.float64)
    y2 = (-s * x + (c * y).astype(np.float32)).astype(np.float32)
    y2 = (y2 + np.float32(h)).astype(np.float32).astype(np.float64)
    inb = ~((x2 < 0) | (x2 > l - 1.0) | (y2 < 0) | (y2 > l - 1.0))
    ii = np.clip(np.floor(x2), 0, l - 1).astype(np.int64)
    jj = np.clip(np.floor(y2), 0, l - 1).astype(np.int64)
    t = x2 - ii
    u = y2 - jj
    k0 = ii + jj * l
    k1 = k0 + 1
    k2 = k0 + l + 1
    k3 = k0 + l
    ex = ii == l - 1
    ey = jj == l - 1
    k1 = np.where(ex, k1 - 1, k1)
    k2 = np.where(ex, k2 - 1, k2)
    k2 = np.where(ey, k2 - l, k2)
    k3 = np.where(ey, k3 - l, k3)
    k0 = np.where(inb, k0, 0)
    k1 = np.clip(np.where(inb, k1, 0), 0, l * l - 1)
    k2 = np.clip(np.where(inb, k2, 0), 0, l * l - 1)
    k3 = np.clip(np.where(inb, k3, 0), 0, l * l - 1)
    flat = T.reshape(n, -1)
    res = (flat[:, k0] * ((1 - t) * (1 - u)) + flat[:, k1] * (t * (1 - u))
           + flat[:, k3] * ((1 - t) * u) + flat[:, k2] * (t * u))
    return np.where(inb[None], res, 0.0)


def soft_mask(l: int, d_m: float) -> np.ndarray:
    """apply_mask factor (GPU_func.cu:229-247): radius 0.75 d_m, 12-px cosine edge."""
    dm = float(f32(1.5 * float(f32(d_m))))
    ehw = 6.0
    j, i = np.mgrid[0:l, 0:l]
    r = hypotf_int(i - l // 2, j - l // 2).astype(np.float64)
    outer = float(f32(f32(dm / 2) + f32(2 * ehw)))
    f = np.ones((l, l))
    f[r > outer] = 0.0
    sel = (r <= outer) & (r >= dm / 2)
    f[sel] = 0.5 * np.cos(PI_REF * (r[sel] - dm / 2) / (2 * ehw)) + 0.5
    return f


def template_spectra(T: np.ndarray, euler3: float, d_m: float,
                     workers: int = 1) -> np.ndarray:
    """rotateTemplate (main.cu:669-716): rotate, mask, zero-mean / unit-variance
    over the full l x l frame, FFT / l^2."""
    n, l, _ = T.shape
    t = rotate_bilinear(T, euler3) * soft_mask(l, d_m)[None]
    flat = t.reshape(n, -1)
    mean = flat.mean(axis=1)
    var = (flat ** 2).mean(axis=1) - mean * mean
    mean_s = np.where(mean != 0, mean, 0.0)
    sd = np.where(var != 0, np.sqrt(np.abs(var)), 1.0)
    t = (t - mean_s[:, None, None]) / sd[:, None, None]
    return _fft2(t, workers) / float(l * l)


# ---------------------------------------------------------------------------
# Micrograph: main.cu:523-655, 758-769
# ---------------------------------------------------------------------------
def hot_pixel_bounds(img: np.ndarray) -> Tuple[np.float32, int, int, bool]:
    """Sequential float32 statistics of init_d_image (main.cu:529-543).

    Returns (avg, up_bound, low_bound, clamp_enabled)."""
    ny, nx = img.shape
    v = img.astype(np.float32).ravel()
    q1 = (v / f32(nx)) / f32(ny)
    q2 = ((v * v) / f32(nx)) / f32(ny)
    s1 = np.add.accumulate(q1)[-1] if v.size else f32(0)
    s2 = np.add.accumulate(q2)[-1] if v.size else f32(0)
    avg = f32(s1)
    with np.errstate(invalid="ignore"):
        var = f32(np.sqrt(f32(f32(s2) - f32(avg * avg))))
    up = f32(avg + f32(f32(6) * var))
    lo = f32(avg - f32(f32(6) * var))
    up_i = int(up) if np.isfinite(up) else 0
    lo_i = int(lo) if np.isfinite(lo) else 0
    return avg, up_i, lo_i, bool(f32(s2) > f32(avg * avg))


def clamp_and_invert(img: np.ndarray, invert: int) -> np.ndarray:
    """Host hot-pixel clamp then optional contrast inversion (main.cu:526-545)."""
    out = img.astype(np.float32).copy()
    avg, up, lo, enabled = hot_pixel_bounds(out)
    if enabled:
        bad = (out > f32(up)) | (out < f32(lo))
        out[bad] = avg
    if invert == 1:
        out = -out
    return out


def preprocess_micrograph(img: np.ndarray, p: Params, ctf: Ctf,
                          workers: int = 1) -> np.ndarray:
    """init_d_image (main.cu:523-586): clamp, invert, FFT/(nx ny), optional phase
    flip + radial whitening + band-pass + Wiener weight (K27, K5, K7), DC = 0,
    unnormalised inverse; returns the real part, float64 (ny, nx)."""
    ny, nx = img.shape
    im = clamp_and_invert(img, p.invert).astype(np.float64)
    F = _fft2(im, workers) / float(nx * ny)
    if p.phase_flip == 1:
        y, x = np.mgrid[0:ny, 0:nx]
        cs = float(f32(p.cs))
        sgn = ctf_ast(x, (y + ny // 2) % ny, nx, ny, p.apix, ctf.dfu, ctf.dfv, ctf.dfdiff,
                      ctf.dfang, ctf.lam, cs, p.ampconst, 0)
        F = F * sgn
        amp2 = F.real ** 2 + F.imag ** 2
        r = shell_index(nx, ny)
        L = max(nx, ny)
        sel = (x <= nx // 2) & (r >= 0) & (r < L // 2)
        ra = np.bincount(r[sel], weights=amp2[sel], minlength=RA_SIZE)
        rb = np.bincount(r[sel], minlength=RA_SIZE).astype(np.float64)
        dx = np.minimum(x, nx - x).astype(np.float64)
        dy = np.minimum(y, ny - y).astype(np.float64)
        apix = float(f32(p.apix))
        ss = np.sqrt((dx * dx / float(nx * nx) + dy * dy / float(ny * ny)) / (apix * apix))
        wsel = (r < L // 2) & (r >= 0)
        v = ctf_ast(x, (y + ny // 2) % ny, nx, ny, p.apix, ctf.dfu, ctf.dfv, ctf.dfdiff,
                    ctf.dfang, ctf.lam, cs, p.ampconst, 2)
        signal = np.exp(p.bfactor * ss * ss + p.bfactor2 * ss + p.bfactor3)
        ncurve = np.exp(p.a * ss * ss + p.b * ss + p.b2)
        rr = np.where(wsel, r, 0)
        with np.errstate(divide="ignore", invalid="ignore"):
            shell_rms = np.sqrt(ra[rr] / rb[rr])
            fac = np.where(wsel, np.sqrt((signal * v * v + ncurve) / signal) / shell_rms, 1.0)
        damp_lim = float(f32(f32(f32(L) * f32(p.apix)) / f32(6)))
        fac = np.where(wsel & (r > damp_lim), fac * np.exp(-100.0 * ss * ss), fac)
        hp = float(f32(f32(f32(L) * f32(p.apix)) / f32(p.highres)))
        lp = float(f32(f32(f32(L) * f32(p.apix)) / f32(p.lowres)))
        fac = fac * _bandpass(r, hp, lp, low_cut=True)
        kk = float(f32(p.kk))
        sig2 = signal / (kk + 1.0)
        nc2 = ncurve / sig2
        fac = np.where(wsel, fac * np.sqrt(1.0 / (nc2 + kk * v * v)), fac)
        F = F * fac
    F[0, 0] = 0.0                                               # K8
    return _ifft2_unnorm(F, workers).real


def split_windows(img: np.ndarray, offx: Sequence[int], offy: Sequence[int],
                  l: int) -> np.ndarray:
    """split_IMG (GPU_func.cu:564-581): window w = i + j*bx; zero beyond the image."""
    ny, nx = img.shape
    out = np.zeros((len(offx) * len(offy), l, l))
    for j, oy in enumerate(offy):
        for i, ox in enumerate(offx):
            blk = img[oy:oy + l, ox:ox + l]
            out[i + j * len(offx), :blk.shape[0], :blk.shape[1]] = blk
    return out


def window_spectra(windows: np.ndarray, p: Params, workers: int = 1) -> np.ndarray:
    """split_normalize_image + fft_on_img (main.cu:588-655, 758-769).

    With phase_flip the reference divides each window's spectrum by
    m = sqrt(sum amp^2 / count^2) over r < l/2, x <= l/2 and round-trips it
    through the inverse FFT; the net effect is W = (FFT(w)/l^2) / m."""
    nw, l, _ = windows.shape
    W = _fft2(windows, workers) / float(l * l)
    if p.phase_flip == 1:
        r = shell_index(l, l)
        y, x = np.mgrid[0:l, 0:l]
        sel = (r >= 0) & (r < l // 2) & (x <= l // 2)
        amp2 = W.real ** 2 + W.imag ** 2
        s = amp2[:, sel].sum(axis=1)
        cnt = float(sel.sum())
        m = np.sqrt(s / (cnt * cnt))
        W = W / np.where(m != 0, m, 1.0)[:, None, None]
    return W


# ---------------------------------------------------------------------------
# Correlation and scoring: GPU_func.cu:584-615, 667-708; main.cu:824-894
# ---------------------------------------------------------------------------
def checker(l: int) -> np.ndarray:
    """compute_corner_CCG's sign pattern (GPU_func.cu:607-614) = (-1)^(l/2) (-1)^(x+y)."""
    y, x = np.mgrid[0:l, 0:l]
    s = np.where((x + y) % 2 == 0, 1.0, -1.0)
    return s if (l // 2) % 2 == 0 else -s


def border_mask(l: int, d_m: float) -> np.ndarray:
    """True where get_peak_and_SUM zeroes the value for the max (GPU_func.cu:681)."""
    q = float(f32(f32(d_m) / f32(4)))
    hi = float(f32(f32(l) - f32(q)))
    y, x = np.mgrid[0:l, 0:l]
    return (x < q) | (x > hi) | (y < q) | (y > hi)


@dataclass
class UnitStats:
    peak: np.ndarray
    pos: np.ndarray
    s1: np.ndarray
    s2: np.ndarray
    sd: np.ndarray
    score: np.ndarray  # NaN where sd <= 0 (reference leaves score unset)


def score_maps(cc: np.ndarray, d_m: float) -> UnitStats:
    """Per-map reduction + host scoring (GPU_func.cu:667-708, main.cu:855-876).

    peak = max(0, max over the non-border pixels), pos = its flat index (0 if
    the peak is 0); sigma excludes the peak: rc = l^2 - 1."""
    n, l, _ = cc.shape
    flat = cc.reshape(n, -1)
    masked = np.where(border_mask(l, d_m).ravel()[None], 0.0, flat)
    mx = masked.max(axis=1)
    am = masked.argmax(axis=1)
    peak = np.where(mx > 0, mx, 0.0)
    pos = np.where(mx > 0, am, 0)
    s1 = flat.sum(axis=1)
    s2 = (flat * flat).sum(axis=1)
    ra = s1 - peak
    rb = s2 - peak * peak
    rc = float(l * l - 1)
    with np.errstate(invalid="ignore", divide="ignore"):
        sd = np.sqrt(rb / rc - (ra / rc) ** 2)
        score = np.where(sd > 0, peak / sd, np.nan)
    return UnitStats(peak, pos, s1, s2, sd, score)


@dataclass
class Pick:
    angle_index: int
    euler3: float
    phi: float
    window_i: int
    window_j: int
    template: int
    cx: float
    cy: float
    score: float


@dataclass
class SearchResult:
    picks: List[Pick]
    angles: List[float]
    offx: List[int]
    offy: List[int]
    l: int
    # dense per-unit tables, shape (n_angles, n_windows, n_templates)
    score: np.ndarray = field(repr=False)
    pos: np.ndarray = field(repr=False)
    peak: np.ndarray = field(repr=False)
    sd: np.ndarray = field(repr=False)
    # per-pixel maximum of cc / sigma over (angle, template) (pixel_thres
    # given): micrograph-sized value (NaN below the threshold) and the
    # winning angle index and template (-1 below the threshold)
    pixel_value: Optional[np.ndarray] = field(default=None, repr=False)
    pixel_angle: Optional[np.ndarray] = field(default=None, repr=False)
    pixel_template: Optional[np.ndarray] = field(default=None, repr=False)


def search(micrograph: np.ndarray, templates_raw: np.ndarray, p: Params,
           ctf: Ctf, ctf_first: Optional[Ctf] = None, prepared: Optional[np.ndarray] = None,
           angles: Optional[Sequence[int]] = None, workers: int = 1,
           dtype=np.complex128, pixel_thres: Optional[float] = None) -> SearchResult:
    """One micrograph of the norm_type 0 search (main.cu:1149-1169, 1230-1257).

    ``templates_raw``: (N, ty, tx) float32 as read from the stack;
    ``ctf_first``: CTF of the first micrograph of the run (templates are
    weighted with it), defaults to ``ctf``; ``prepared``: precomputed output
    of :func:`prepare_templates`; ``angles``: optional subset of angle
    indices (the dense tables then hold NaN elsewhere).

    ``pixel_thres`` (no reference counterpart): also build the per-pixel
    maximum over (angle, template) of every map normalised by its own sigma
    (the score's sigma, without the peak), over the non-border pixels the
    score's maximum looks at, each map pixel placed at its particle centre
    (window offset + fftshifted index) and the windows merged by maximum;
    values below ``pixel_thres`` are left out.  Among equal values the first
    in (angle, window, template) order wins."""
    ny, nx = micrograph.shape
    n, ty, tx = templates_raw.shape
    l = adjust_padding_size(p.padding_size, tx, ty)
    if ctf_first is None:
        ctf_first = ctf
    T = prepared if prepared is not None else prepare_templates(templates_raw, p, l, ctf_first, workers)
    img = preprocess_micrograph(micrograph, p, ctf, workers)
    offx = window_offsets(nx, l, p.overlap)
    offy = window_offsets(ny, l, p.overlap)
    bx, by = len(offx), len(offy)
    W = window_spectra(split_windows(img, offx, offy, l), p, workers).astype(dtype)
    chk = checker(l)
    angs = angle_list(p.phi_step)
    sel_angles = range(len(angs)) if angles is None else angles
    na, nw = len(angs), bx * by
    tab = {k: np.full((na, nw, n), np.nan) for k in ("score", "peak", "sd")}
    tab_pos = np.full((na, nw, n), -1, dtype=np.int64)
    picks: List[Pick] = []
    d_m = float(f32(p.d_m))
    thres = f32(p.thres)
    if pixel_thres is not None:
        pix_v = np.full((ny, nx), -np.inf)
        pix_a = np.full((ny, nx), -1, dtype=np.int64)
        pix_t = np.full((ny, nx), -1, dtype=np.int64)
        inner = ~border_mask(l, p.d_m)
    for ai in sel_angles:
        e = angs[ai]
        TS = template_spectra(T, e, p.d_m, workers).astype(dtype)
        TSc = np.conj(TS) * chk[None]
        for j in range(by):
            for i in range(bx):
                w = i + j * bx
                cc = _ifft2_unnorm(W[w][None] * TSc, workers).real
                st = score_maps(cc, p.d_m)
                tab["score"][ai, w] = st.score
                tab["peak"][ai, w] = st.peak
                tab["sd"][ai, w] = st.sd
                tab_pos[ai, w] = st.pos
                if pixel_thres is not None:
                    for J in range(n):
                        if not (np.isfinite(st.score[J]) and st.sd[J] > 0):
                            continue
                        z = np.where(inner, cc[J] / st.sd[J], -np.inf)
                        sub_v = pix_v[offy[j]:offy[j] + l, offx[i]:offx[i] + l]
                        win = (z >= pixel_thres) & (z > sub_v)
                        sub_v[win] = z[win]
                        pix_a[offy[j]:offy[j] + l, offx[i]:offx[i] + l][win] = ai
                        pix_t[offy[j]:offy[j] + l, offx[i]:offx[i] + l][win] = J
                for J in range(n):
                    sc = st.score[J]
                    if not np.isfinite(sc) or f32(sc) < thres:
                        continue
                    cx = float(offx[i] + int(st.pos[J]) % l)
                    cy = float(offy[j] + int(st.pos[J]) // l)
                    if cx >= d_m and cx < nx - d_m and cy >= d_m and cy < ny - d_m:
                        picks.append(Pick(ai, float(e), float(printed_phi(e)), i, j, J,
                                          cx, cy, float(sc)))
    res = SearchResult(picks, [float(a) for a in angs], offx, offy, l,
                       tab["score"], tab_pos, tab["peak"], tab["sd"])
    if pixel_thres is not None:
        res.pixel_value = np.where(np.isfinite(pix_v), pix_v, np.nan)
        res.pixel_angle, res.pixel_template = pix_a, pix_t
    return res


@dataclass
class BlockPick:
    angle_index: int
    euler3: float
    phi: float
    window_i: int
    window_j: int
    template: int
    block: int
    cx: float
    cy: float
    score: float


def search_norm1(micrograph: np.ndarray, templates_raw: np.ndarray, p: Params, ctf: Ctf,
                 ctf_first: Optional[Ctf] = None, prepared: Optional[np.ndarray] = None,
                 workers: int = 1):
    """norm_type 1 (main.cu:1170-1229): every correlation value is z-scored
    against the mean and standard deviation of that window pixel over all
    templates and angles (first sweep: compute_CCG_sum / add_CCG_to_sum /
    set_CCG_mean, main.cu:724-756, GPU_func.cu:617-646), then in a second
    sweep each 1024-element block of the z-scored maps reports its maximum
    and position (update_CCG + get_peak_pos, GPU_func.cu:648-662, 711-745; no
    border mask) and a line is written when it reaches the threshold and the
    centre lies at least d_m inside the micrograph (main.cu:800-817).
    Returns (picks in reference order, per-window mean, per-window std)."""
    ny, nx = micrograph.shape
    n, ty, tx = templates_raw.shape
    l = adjust_padding_size(p.padding_size, tx, ty)
    if (l * l) % 1024:
        raise ValueError("norm_type 1 needs l*l to be a multiple of 1024")
    if ctf_first is None:
        ctf_first = ctf
    T = prepared if prepared is not None else prepare_templates(templates_raw, p, l, ctf_first, workers)
    img = preprocess_micrograph(micrograph, p, ctf, workers)
    offx = window_offsets(nx, l, p.overlap)
    offy = window_offsets(ny, l, p.overlap)
    bx, by = len(offx), len(offy)
    W = window_spectra(split_windows(img, offx, offy, l), p, workers)
    chk = checker(l)
    angs = angle_list(p.phi_step)
    l2 = float(l * l)
    s1 = np.zeros((bx * by, l, l))
    s2 = np.zeros((bx * by, l, l))
    spectra = []
    for e in angs:
        TSc = np.conj(template_spectra(T, e, p.d_m, workers)) * chk[None]
        spectra.append(TSc)
        for w in range(bx * by):
            cur = _ifft2_unnorm(W[w][None] * TSc, workers).real / l2
            s1[w] += cur.sum(axis=0)
            s2[w] += (cur * cur).sum(axis=0)
    total = float(n * len(angs))
    avg = s1 / total
    with np.errstate(invalid="ignore"):
        std = np.sqrt(s2 / total - avg * avg)
    nblk = (l * l) // 1024
    d_m = float(f32(p.d_m))
    thres = f32(p.thres)
    picks: List[BlockPick] = []
    for ai, e in enumerate(angs):
        for j in range(by):
            for i in range(bx):
                w = i + j * bx
                cur = _ifft2_unnorm(W[w][None] * spectra[ai], workers).real / l2
                with np.errstate(invalid="ignore", divide="ignore"):
                    z = np.where(std[w][None] > 0, (cur - avg[w][None]) / std[w][None], 0.0)
                zb = z.reshape(n, nblk, 1024)
                mx = zb.max(axis=2)
                am = zb.argmax(axis=2)
                for J in range(n):
                    for b in range(nblk):
                        if f32(mx[J, b]) < thres:
                            continue
                        pos = b * 1024 + int(am[J, b])
                        cx = float(offx[i] + pos % l)
                        cy = float(offy[j] + pos // l)
                        if cx >= d_m and cx < nx - d_m and cy >= d_m and cy < ny - d_m:
                            picks.append(BlockPick(ai, float(e), float(printed_phi(e)), i, j, J, b,
                                                   cx, cy, float(mx[J, b])))
    return picks, avg, std


def params_from_config(cfg) -> Params:
    """Params from a parsed config object with the reference's field names."""
    return Params(apix=cfg.apix, phi_step=cfg.phi_step, kk=cfg.kk, energy=cfg.energy,
                  cs=cfg.cs, highres=cfg.highres, lowres=cfg.lowres, d_m=cfg.d_m,
                  first=cfg.first, last=cfg.last, thres=cfg.thres,
                  padding_size=cfg.padding_size, phase_flip=cfg.phase_flip,
                  overlap=cfg.overlap, invert=cfg.invert, norm_type=cfg.norm_type)


def run_config(config_path: str, workers: int = 1, return_results: bool = False):
    """Whole-run restatement of ``main`` for norm_type 0 (main.cu:1025-1269):
    returns the output lines the reference writes to its .lst file.

    Paths in the config are resolved relative to the current directory, as
    the reference does.  File parsing uses the package's reference-format
    readers (gisspa_b200.formats), which the golden tests pin separately."""
    from gisspa_b200 import formats
    cfg = formats.read_config(config_path)
    p = params_from_config(cfg)
    eul = formats.read_euler(cfg.eulerf)
    raw0 = formats.read_mrc(cfg.temp2d, 0)
    ty, tx = raw0.shape
    n = eul.shape[0]
    raw = np.stack([formats.read_mrc(cfg.temp2d, k) for k in range(n)])
    l = adjust_padding_size(p.padding_size, tx, ty)
    first = formats.read_lst_entry(cfg.inlst, cfg.first)
    # ds uses the configured window size: main.cu:155 runs before main.cu:1116
    ctf0 = make_ctf(p, first.defocus, first.dfdiff, first.dfang, p.padding_size)
    T = prepare_templates(raw, p, l, ctf0, workers)
    lines: List[str] = []
    results = []
    for m in range(cfg.first, cfg.last):
        ent = formats.read_lst_entry(cfg.inlst, m)
        img = formats.read_mrc(ent.path, ent.nn)
        ctf = make_ctf(p, ent.defocus, ent.dfdiff, ent.dfang, l)
        if p.norm_type == 1:
            picks, _, _ = search_norm1(img, raw, p, ctf, ctf0, prepared=T, workers=workers)
            results.append(picks)
        else:
            res = search(img, raw, p, ctf, ctf0, prepared=T, workers=workers)
            results.append(res)
            picks = res.picks
        for pk in picks:
            lines.append(format_pick_line(ent.nn, ent.path, ctf, float(eul[pk.template, 0]),
                                          float(eul[pk.template, 1]), pk))
    return (lines, results) if return_results else lines


def format_pick_line(nn: int, path: str, ctf: Ctf, euler_alt: float, euler_az: float,
                     pick: Pick) -> str:
    """writeScoreToDisk line (main.cu:985-987); float32 values through %f."""
    vals = (float(f32(-f32(ctf.defocus))), float(f32(ctf.dfdiff)), float(f32(ctf.dfang)),
            float(f32(euler_alt)), float(f32(euler_az)), float(f32(pick.phi)),
            float(f32(pick.cx)), float(f32(pick.cy)), float(f32(pick.score)))
    return ("%d\t%s\tdefocus=%f\tdfdiff=%f\tdfang=%f\teuler=%f,%f,%f\tcenter=%f,%f\tscore=%f\n"
            % ((nn, path) + vals))
