"""FP64 reference of the per-pick refinement objective and its gradient.

TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and bench.py's
baseline legs may import this module; the product never does.

The objective has no reference counterpart (the reference only scores a
fixed grid of angles and pixels).  It continues the reference's own score
off the grid, with the same steps in the same order:

  B     = FFT(b) / l^2                     b: the template after padding, edge
                                           normalisation and whitening
                                           (main.cu:182-431), real l x l
  F1    = B * w(k; defocus, dfdiff, dfang) band-pass x |CTF| Wiener weight
                                           (GPU_func.cu:249-290)
  F2    = F1 / a,  a = sqrt(sum_sel |F1|^2) / cnt     (K12 + K14, main.cu:447-458)
  t     = Re IFFT(F2)                      (main.cu:463)
  t_m   = mask * bilinear_rotate(t, e)     (GPU_func.cu:496-560, 229-247)
  t_n   = (t_m - mean) / sd                over the full frame (main.cu:697-710)
  F     = FFT(t_n) / l^2
  c     = Re sum_k W(k) conj(F(k)) exp(2 pi i k.(x0 + d) / l)   k signed
  sigma = sqrt(sum_k |W(k)|^2 |F(k)|^2)    the map's standard deviation by
                                           Parseval (the window spectrum has no
                                           DC term, so the map has zero mean)
  s     = sgn * c / sigma,  sgn = (-1)^(l/2) as in the fftshift of the search

At d = 0, the grid angle and the CTF of the weight this is the search's score
up to the peak's own contribution to sigma (relative O(peak^2 / (l^2 sigma^2))).
x0 is the unshifted map position of the pick (pos - l/2 per axis, mod l).
Rotation follows the reference's bilinear sampling, including its edge index
rules, with exact (not float-rounded) source coordinates.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from . import gisspa_oracle as G

PI_REF = 3.141592654


@dataclass
class WeightConsts:
    """Constants of the template weight (reference Parameters fields)."""
    apix: float
    l: int
    highres: float
    lowres: float
    kk: float
    cs: float
    ampconst: float
    lam: float          # electron wavelength, A
    ds: float           # 1 / (apix * configured window)
    a: float = -9.32
    b: float = 2.65
    b2: float = 0.01908
    bfactor: float = -78.7757
    bfactor2: float = -12.9121
    bfactor3: float = 1.28732


def _grids(l: int):
    y, x = np.mgrid[0:l, 0:l]
    return y, x


def weight_parts(wc: WeightConsts):
    """theta-independent pieces of the weight on the l x l grid (float64):
    band factor, in-band selector, ss, atan2 angle, noise curve."""
    l = wc.l
    y, x = _grids(l)
    rf = G.hypotf_int(np.minimum(y, l - y), np.minimum(x, l - x)).astype(np.float64)
    r_round = (np.floor(rf + 0.5) - 1).astype(np.int64)
    hp = float(G.f32(G.f32(G.f32(l) * G.f32(wc.apix)) / G.f32(wc.highres)))
    lp = float(G.f32(G.f32(G.f32(l) * G.f32(wc.apix)) / G.f32(wc.lowres)))
    band = G._bandpass(r_round, hp, lp, low_cut=False)
    wsel = (r_round < l // 2) & (r_round >= 0)
    ss_w = rf * float(G.f32(wc.ds))
    # CTF geometry: ctf_ast(x, (y + l/2) % l) with its own folding
    x1 = x.copy()
    y1 = (y + l // 2) % l
    y1 = np.where(x1 > l // 2, l - y1, y1)
    x1 = np.minimum(x1, l - x1)
    dx = x1.astype(np.float64)
    dy = (y1 - l // 2).astype(np.float64)
    apix = float(np.float32(wc.apix))
    ss = (dx * dx / float(l * l) + dy * dy / float(l * l)) / (apix * apix)
    ag = np.arctan2(dy, dx)
    kk = float(np.float32(wc.kk))
    signal = np.exp(wc.bfactor * ss_w * ss_w + wc.bfactor2 * ss_w + wc.bfactor3) / (kk + 1.0)
    ncurve = np.exp(wc.a * ss_w * ss_w + wc.b * ss_w + wc.b2) / signal
    return band, wsel, ss, ag, ncurve


def weight_torch(wc: WeightConsts, theta: torch.Tensor, parts) -> torch.Tensor:
    """w(k; theta) with theta = (defocus um, dfdiff um, dfang deg), float64."""
    band, wsel, ss, ag, ncurve = (torch.as_tensor(p) for p in parts)
    D = -theta[0]
    dfdiff = theta[1]
    ang = theta[2] * PI_REF / 180.0
    df_ast = D + dfdiff * torch.cos(2.0 * (ang - ag))
    lam = wc.lam
    gamma = -2.0 * PI_REF * (float(np.float32(wc.cs)) * 2.5e6 * lam ** 3 * ss * ss + df_ast * 5000.0 * lam * ss)
    a = float(np.float32(wc.ampconst))
    v = math.sqrt(1.0 - a * a) * torch.sin(gamma) + a * torch.cos(gamma)
    v = torch.abs(v)
    kk = float(np.float32(wc.kk))
    w = v * torch.sqrt(1.0 / (ncurve + kk * v * v))
    return band * torch.where(wsel, w, torch.ones_like(w))


def rotate_torch(t: torch.Tensor, e: torch.Tensor) -> torch.Tensor:
    """Bilinear rotation of rotate_subIMG with the reference's index rules;
    differentiable in t and e (exact source coordinates)."""
    l = t.shape[-1]
    h = l // 2
    j, i = np.mgrid[0:l, 0:l]
    x = torch.as_tensor((i - h).astype(np.float64))
    y = torch.as_tensor((j - h).astype(np.float64))
    ang = e * PI_REF / 180.0
    c, s = torch.cos(ang), torch.sin(ang)
    x2 = c * x + s * y + h
    y2 = -s * x + c * y + h
    inb = ~((x2 < 0) | (x2 > l - 1.0) | (y2 < 0) | (y2 > l - 1.0))
    ii = torch.clamp(torch.floor(x2.detach()), 0, l - 1).long()
    jj = torch.clamp(torch.floor(y2.detach()), 0, l - 1).long()
    tt = x2 - ii
    uu = y2 - jj
    k0 = ii + jj * l
    k1 = k0 + 1
    k2 = k0 + l + 1
    k3 = k0 + l
    ex = ii == l - 1
    ey = jj == l - 1
    k1 = torch.where(ex, k1 - 1, k1)
    k2 = torch.where(ex, k2 - 1, k2)
    k2 = torch.where(ey, k2 - l, k2)
    k3 = torch.where(ey, k3 - l, k3)
    zero = torch.zeros_like(k0)
    k0 = torch.where(inb, k0, zero)
    k1 = torch.clamp(torch.where(inb, k1, zero), 0, l * l - 1)
    k2 = torch.clamp(torch.where(inb, k2, zero), 0, l * l - 1)
    k3 = torch.clamp(torch.where(inb, k3, zero), 0, l * l - 1)
    flat = t.reshape(-1)
    res = (flat[k0] * ((1 - tt) * (1 - uu)) + flat[k1] * (tt * (1 - uu))
           + flat[k3] * ((1 - tt) * uu) + flat[k2] * (tt * uu))
    return torch.where(inb, res, torch.zeros_like(res))


def signed_freq(l: int) -> np.ndarray:
    k = np.arange(l)
    return np.where(k < l // 2 + (l % 2), k, k - l).astype(np.float64)


def score_torch(b: torch.Tensor, W: torch.Tensor, x0: tuple, e: torch.Tensor, d: torch.Tensor,
                theta: torch.Tensor, wc: WeightConsts, parts, mask: np.ndarray) -> torch.Tensor:
    """The objective s (see module docstring), float64, differentiable in b,
    e, d and theta.  W: complex128 window spectrum (l x l); x0 = (X0, Y0)."""
    l = b.shape[-1]
    L2 = float(l * l)
    B = torch.fft.fft2(b) / L2
    F1 = B * weight_torch(wc, theta, parts)
    _, wsel, _, _, _ = parts
    y, x = _grids(l)
    sel = torch.as_tensor(((x <= l // 2) & wsel))
    cnt = float(sel.sum())
    a = torch.sqrt((F1.real ** 2 + F1.imag ** 2)[sel].sum()) / cnt
    t = torch.fft.ifft2(F1 / a).real * L2
    tm = rotate_torch(t, e) * torch.as_tensor(mask)
    mu = tm.mean()
    var = (tm * tm).mean() - mu * mu
    tn = (tm - mu) / torch.sqrt(var)
    F = torch.fft.fft2(tn) / L2
    kf = torch.as_tensor(signed_freq(l))
    ph = 2.0 * math.pi * (kf[None, :] * (x0[0] + d[0]) + kf[:, None] * (x0[1] + d[1])) / l
    E = torch.complex(torch.cos(ph), torch.sin(ph))
    Gk = W * torch.conj(F)
    c = (Gk * E).real.sum()
    sigma = torch.sqrt(((W.real ** 2 + W.imag ** 2) * (F.real ** 2 + F.imag ** 2)).sum())
    sgn = 1.0 if (l // 2) % 2 == 0 else -1.0
    return sgn * c / sigma


def score_and_grad(b, W, x0, e, d, theta, wc, parts, mask):
    """(s, ds/de, ds/dd (2), ds/dtheta (3), ds/db (l x l)) in float64."""
    bt = torch.tensor(b, dtype=torch.float64, requires_grad=True)
    Wt = torch.tensor(W, dtype=torch.complex128)
    et = torch.tensor(float(e), dtype=torch.float64, requires_grad=True)
    dt = torch.tensor(np.asarray(d, dtype=np.float64), requires_grad=True)
    th = torch.tensor(np.asarray(theta, dtype=np.float64), requires_grad=True)
    s = score_torch(bt, Wt, x0, et, dt, th, wc, parts, mask)
    s.backward()
    return (float(s), float(et.grad), dt.grad.numpy().copy(), th.grad.numpy().copy(),
            bt.grad.numpy().copy())


def template_base(raw: np.ndarray, l: int) -> np.ndarray:
    """b for every template: padding, edge normalisation and the radial-shell
    whitening of handleTemplate (main.cu:182-431), before the CTF weight;
    real (N, l, l) float64.  FFT(b) / l^2 times the weight, amplitude
    normalised and inverse transformed gives gisspa_oracle.prepare_templates."""
    T = G.edge_normalize(G.pad_templates(raw, l))
    n = T.shape[0]
    F = np.fft.fft2(T, axes=(-2, -1)) / float(l * l)
    amp2 = F.real ** 2 + F.imag ** 2
    r = G.shell_index(l, l)
    y, x = np.mgrid[0:l, 0:l]
    sel = (x <= l // 2) & (r >= 0) & (r < l // 2)
    shell_ok = (r >= 0) & (r < l // 2)
    out = np.empty((n, l, l))
    for k in range(n):
        ra = np.bincount(r[sel], weights=amp2[k][sel], minlength=l // 2)
        rb = np.bincount(r[sel], minlength=l // 2).astype(np.float64)
        with np.errstate(divide="ignore", invalid="ignore"):
            fac = 1.0 / np.sqrt(ra / rb)
        wk = np.ones((l, l))
        wk[shell_ok] = fac[r[shell_ok]]
        out[k] = np.fft.ifft2(F[k] * wk).real * float(l * l)
    return out


def weight_consts(p, l: int, ctf) -> WeightConsts:
    """WeightConsts from oracle Params and a Ctf (its lam and ds)."""
    return WeightConsts(apix=p.apix, l=l, highres=p.highres, lowres=p.lowres, kk=p.kk, cs=p.cs,
                        ampconst=p.ampconst, lam=ctf.lam, ds=ctf.ds, a=p.a, b=p.b, b2=p.b2,
                        bfactor=p.bfactor, bfactor2=p.bfactor2, bfactor3=p.bfactor3)
