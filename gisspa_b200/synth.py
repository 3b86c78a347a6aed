"""Seeded synthetic inputs for the GisSPA search (micrographs, template stack,
Euler file, input list, config).

No public dataset is used: the density is a sum of isotropic 3D Gaussian
blobs whose projections are analytic 2D Gaussians (a 3D Gaussian of width
sigma projects to a 2D Gaussian of amplitude sqrt(2 pi) sigma), so templates
and particles are exact.  Particles are projections of the same density at
template orientations, rotated in plane by an angle of the search grid,
CTF-modulated in Fourier space, scaled to the requested SNR inside the
particle disc and added to Gaussian noise (white, or coloured with power
~ 1/f^alpha).  Everything is a function of the seed.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import formats

PI = math.pi


@dataclass
class Density:
    centers: np.ndarray  # (B, 3) px, relative to the particle centre
    sigmas: np.ndarray   # (B,)
    weights: np.ndarray  # (B,)


def make_density(rng: np.random.Generator, n_blobs: int, radius: float,
                 sigma_range=(2.0, 5.0)) -> Density:
    """Blob centres uniform in a ball, widths uniform in ``sigma_range``."""
    d = rng.standard_normal((n_blobs, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = radius * rng.random(n_blobs) ** (1.0 / 3.0)
    return Density(d * r[:, None], rng.uniform(*sigma_range, n_blobs), np.ones(n_blobs))


def random_views(rng: np.random.Generator, n: int) -> np.ndarray:
    """(n, 2) (alt, az) degrees of directions uniform on the sphere (phi = 0)."""
    alt = np.degrees(np.arccos(rng.uniform(-1.0, 1.0, n)))
    az = rng.uniform(0.0, 360.0, n)
    return np.stack([alt, az], axis=1).astype(np.float32)


def eman_matrix(alt_deg: float, az_deg: float, phi_deg: float = 0.0) -> np.ndarray:
    """EMAN (alt, az, phi) rotation; its decomposition is alt = acos(m8),
    az = atan2(m6, -m7), phi = atan2(m2, m5)."""
    a, z, p = (math.radians(v) for v in (alt_deg, az_deg, phi_deg))
    ca, sa, cz, sz, cp, sp = math.cos(a), math.sin(a), math.cos(z), math.sin(z), math.cos(p), math.sin(p)
    return np.array([
        [cp * cz - ca * sz * sp, cp * sz + ca * cz * sp, sa * sp],
        [-sp * cz - ca * sz * cp, -sp * sz + ca * cz * cp, sa * cp],
        [sa * sz, -sa * cz, ca]])


def projected_blobs(den: Density, alt: float, az: float) -> Tuple[np.ndarray, np.ndarray]:
    """2D centres (x, y) and amplitudes of the projection along z after rotation."""
    R = eman_matrix(alt, az)
    c = den.centers @ R.T
    amp = den.weights * math.sqrt(2.0 * PI) * den.sigmas
    return c[:, :2], amp


def render_gaussians(centers_xy: np.ndarray, amps: np.ndarray, sigmas: np.ndarray,
                     size: int, dtype=np.float64) -> np.ndarray:
    """Separable render of sum_b amp_b exp(-|p - c_b|^2 / (2 s_b^2)) on a size^2
    grid whose centre pixel (size//2, size//2) is the origin."""
    g = np.arange(size, dtype=np.float64) - size // 2
    gx = np.exp(-((g[None, :] - centers_xy[:, 0:1]) ** 2) / (2 * sigmas[:, None] ** 2))
    gy = np.exp(-((g[None, :] - centers_xy[:, 1:2]) ** 2) / (2 * sigmas[:, None] ** 2))
    return (gy.T.astype(dtype) @ (amps[:, None] * gx).astype(dtype)).astype(np.float64)


def render_gaussians_batch(centers_xy: np.ndarray, amps: np.ndarray, sigmas: np.ndarray,
                           size: int) -> np.ndarray:
    """float32 batched version of :func:`render_gaussians` on CPU threads:
    centers_xy (K, B, 2), amps (K, B) -> (K, size, size)."""
    import torch
    g = torch.arange(size, dtype=torch.float32) - size // 2
    c = torch.from_numpy(np.ascontiguousarray(centers_xy, dtype=np.float32))
    a = torch.from_numpy(np.ascontiguousarray(amps, dtype=np.float32))
    s2 = torch.from_numpy(np.asarray(2.0 * sigmas ** 2, dtype=np.float32))[None, :, None]
    gx = torch.exp(-((g[None, None, :] - c[:, :, 0:1]) ** 2) / s2) * a[:, :, None]
    gy = torch.exp(-((g[None, None, :] - c[:, :, 1:2]) ** 2) / s2)
    return torch.bmm(gy.transpose(1, 2), gx).numpy()


def jittered_grid(rng: np.random.Generator, nx: int, ny: int, count: int, margin: float,
                  min_dist: float) -> List[Tuple[int, int]]:
    """``count`` positions >= ``margin`` from the edges and >= ``min_dist``
    apart: one per cell of a grid of pitch min_dist + 2 j, jittered by +-j."""
    jit = 8
    pitch = int(math.ceil(min_dist)) + 2 * jit
    xs = np.arange(int(math.ceil(margin)) + jit, nx - int(math.ceil(margin)) - jit, pitch)
    ys = np.arange(int(math.ceil(margin)) + jit, ny - int(math.ceil(margin)) - jit, pitch)
    cells = [(x, y) for y in ys for x in xs]
    pick = rng.permutation(len(cells))[:count]
    out = []
    for k in pick:
        x, y = cells[k]
        out.append((int(x + rng.integers(-jit, jit + 1)), int(y + rng.integers(-jit, jit + 1))))
    return out


def ctf_value(size: int, apix: float, defocus_um: float, dfdiff_um: float, dfang_deg: float,
              voltage_kv: float = 300.0, cs_mm: float = 2.7, ampconst: float = 0.07) -> np.ndarray:
    """Signed CTF on an unshifted size^2 FFT grid, underfocus positive in um,
    astigmatism half-difference ``dfdiff`` at angle ``dfang``; same sign and
    astigmatism conventions as the search's own CTF model, so a phase-flipped
    particle correlates positively with its template."""
    lam = 12.2639 / math.sqrt(voltage_kv * 1000.0 + 0.97845 * voltage_kv * voltage_kv)
    f = np.fft.fftfreq(size) / apix
    fy, fx = np.meshgrid(f, f, indexing="ij")
    s2 = fx * fx + fy * fy
    ang = np.arctan2(fy, fx)
    df = (defocus_um - dfdiff_um * np.cos(2 * (ang - math.radians(dfang_deg)))) * 1e4
    gamma = PI * lam * df * s2 - 0.5 * PI * cs_mm * 1e7 * lam ** 3 * s2 * s2
    return math.sqrt(1 - ampconst ** 2) * np.sin(gamma) + ampconst * np.cos(gamma)


def coloured_noise(rng: np.random.Generator, ny: int, nx: int, alpha: float) -> np.ndarray:
    """Unit-variance Gaussian noise with power ~ 1/f^alpha (white for alpha 0)."""
    n = rng.standard_normal((ny, nx))
    if alpha == 0:
        return n
    F = np.fft.rfft2(n)
    fy = np.fft.fftfreq(ny)[:, None]
    fx = np.fft.rfftfreq(nx)[None, :]
    f = np.sqrt(fx * fx + fy * fy)
    f[0, 0] = 1.0
    F *= f ** (-alpha / 2.0)
    F[0, 0] = 0.0
    out = np.fft.irfft2(F, s=(ny, nx))
    return out / out.std()


@dataclass
class Particle:
    x: int
    y: int
    template: int
    angle_index: int


@dataclass
class Micrograph:
    image: np.ndarray          # (ny, nx) float32
    defocus: float
    dfdiff: float
    dfang: float
    particles: List[Particle]


@dataclass
class Dataset:
    templates: np.ndarray      # (N, t, t) float32
    views: np.ndarray          # (N, 2) float32 alt, az
    micrographs: List[Micrograph]
    params: Dict[str, object]  # config keys (reference names)


def place_particles(rng: np.random.Generator, nx: int, ny: int, count: int, margin: float,
                    min_dist: float, max_tries: int = 200000) -> List[Tuple[int, int]]:
    pts: List[Tuple[int, int]] = []
    tries = 0
    while len(pts) < count and tries < max_tries:
        tries += 1
        x = int(rng.integers(int(math.ceil(margin)), int(nx - margin)))
        y = int(rng.integers(int(math.ceil(margin)), int(ny - margin)))
        if all((x - a) ** 2 + (y - b) ** 2 >= min_dist ** 2 for a, b in pts):
            pts.append((x, y))
    return pts


def make_dataset(seed: int, *, nx: int, ny: int, n_templates: int, tsize: int,
                 n_particles: int, snr: float, n_blobs: int, ball_radius: float,
                 phistep: float, diameter: float, window: int, overlap: int,
                 apix: float = 1.0, defocus=(1.5, 1.5), astig_A: float = 0.0,
                 noise_alpha: float = 0.0, n_micrographs: int = 1,
                 sizes: Optional[Sequence[Tuple[int, int]]] = None,
                 hot_pixels: int = 0, threshold: float = 7.0, phase_flip: int = 1,
                 invert: int = 0, highres: float = 8.0, lowres: float = 100.0,
                 kk: float = 3.0, fast: bool = False) -> Dataset:
    """``fast`` renders in float32 with a particle box of 1.5 x the template
    size (instead of the next power of two); used for the large workloads."""
    rng = np.random.default_rng(seed)
    den = make_density(rng, n_blobs, ball_radius)
    views = random_views(rng, n_templates)
    tmpl = np.empty((n_templates, tsize, tsize), dtype=np.float32)
    if fast:
        for k0 in range(0, n_templates, 250):
            proj = [projected_blobs(den, float(views[k, 0]), float(views[k, 1]))
                    for k in range(k0, min(n_templates, k0 + 250))]
            tmpl[k0:k0 + len(proj)] = render_gaussians_batch(
                np.stack([c for c, _ in proj]), np.stack([a for _, a in proj]), den.sigmas, tsize)
    else:
        for k in range(n_templates):
            c, a = projected_blobs(den, float(views[k, 0]), float(views[k, 1]))
            tmpl[k] = render_gaussians(c, a, den.sigmas, tsize).astype(np.float32)
    n_angles = int(math.ceil(360.0 / phistep - 1e-9))
    mics: List[Micrograph] = []
    box = (int(math.ceil(tsize * 0.75)) * 2) if fast else int(2 ** math.ceil(math.log2(tsize * 1.5)))
    for m in range(n_micrographs):
        mx, my = (sizes[m] if sizes is not None else (nx, ny))
        img = coloured_noise(rng, my, mx, noise_alpha)
        d0 = float(rng.uniform(*defocus)) if defocus[0] != defocus[1] else float(defocus[0])
        dd = float(rng.uniform(0.0, astig_A)) / 2.0 / 1e4 if astig_A > 0 else 0.0
        da = float(rng.uniform(0.0, 180.0)) if astig_A > 0 else 0.0
        ctf = ctf_value(box, apix, d0, dd, da)
        if fast:
            pts = jittered_grid(rng, mx, my, n_particles, diameter + box // 2, 2 * ball_radius)
        else:
            pts = place_particles(rng, mx, my, n_particles, diameter + box // 2, diameter)
        parts: List[Particle] = []
        sig = np.zeros((my, mx))
        disc_vals = []
        choice = [(int(rng.integers(0, n_templates)), int(rng.integers(0, n_angles))) for _ in pts]
        rendered = None
        if fast and pts:
            cs_, as_ = [], []
            for (J, ai) in choice:
                e = math.radians(ai * phistep)
                c, s = math.cos(e), math.sin(e)
                q, a = projected_blobs(den, float(views[J, 0]), float(views[J, 1]))
                cs_.append(np.stack([c * q[:, 0] - s * q[:, 1], s * q[:, 0] + c * q[:, 1]], axis=1))
                as_.append(a)
            rendered = render_gaussians_batch(np.stack(cs_), np.stack(as_), den.sigmas, box)
        for idx, (x, y) in enumerate(pts):
            J, ai = choice[idx]
            if rendered is not None:
                p = rendered[idx].astype(np.float64)
            else:
                e = math.radians(ai * phistep)
                c, s = math.cos(e), math.sin(e)
                q, a = projected_blobs(den, float(views[J, 0]), float(views[J, 1]))
                # the search rotates template J by e with source (c x + s y, -s x + c y):
                # the matching particle has its blob centres at (c qx - s qy, s qx + c qy)
                rc = np.stack([c * q[:, 0] - s * q[:, 1], s * q[:, 0] + c * q[:, 1]], axis=1)
                p = render_gaussians(rc, a, den.sigmas, box)
            p = np.fft.ifft2(np.fft.fft2(np.fft.ifftshift(p)) * ctf).real
            p = np.fft.fftshift(p)
            x0, y0 = x - box // 2, y - box // 2
            sig[y0:y0 + box, x0:x0 + box] += p
            yy, xx = np.mgrid[0:box, 0:box]
            disc = (xx - box // 2) ** 2 + (yy - box // 2) ** 2 <= (diameter / 2) ** 2
            disc_vals.append(p[disc])
            parts.append(Particle(x, y, J, ai))
        if disc_vals:
            sv = np.concatenate(disc_vals).var()
            scale = math.sqrt(snr * img.var() / sv) if sv > 0 else 0.0
            img = img + scale * sig
        if hot_pixels:
            hp = rng.integers(0, my * mx, hot_pixels)
            img.ravel()[hp] = rng.choice([-1.0, 1.0], hot_pixels) * 60.0
        mics.append(Micrograph(img.astype(np.float32), d0, dd, da, parts))
    params = {
        "angpix": apix, "phistep": phistep, "kk": kk, "energy": 300, "cs": 2.7,
        "Highres": highres, "Lowres": lowres, "diameter": diameter, "threshold": threshold,
        "window_size": window, "overlap": overlap, "phase_flip": phase_flip,
        "norm_type": 0, "invert": invert, "GPU_ID": 0, "first": 0,
        "last": n_micrographs,
    }
    return Dataset(tmpl, views, mics, params)


# ---------------------------------------------------------------------------
# The workloads the benchmark configurations describe
# ---------------------------------------------------------------------------
def config_small(seed: int = 0) -> Dict[str, object]:
    """1024^2 micrograph, 20 particles at SNR 0.05, 50 templates 128^2 from a
    200-blob density in a 40-px ball, 5 deg in-plane step, window 512 with
    overlap 128, defocus 1.5 um."""
    return dict(seed=seed, nx=1024, ny=1024, n_templates=50, tsize=128, n_particles=20,
                snr=0.05, n_blobs=200, ball_radius=40.0, phistep=5.0, diameter=90.0,
                window=512, overlap=128, defocus=(1.5, 1.5), threshold=7.0)


BATCH_SIZES = ((3838, 3710), (4096, 4096), (5760, 4092))


def config_batch(seed: int = 2, n_micrographs: int = 32) -> Dict[str, object]:
    """Uneven batch: n micrographs with sizes drawn (seeded) from 3838 x 3710,
    4096 x 4096 and 5760 x 4092, 250 particles each at SNR 0.03, per-micrograph
    defocus 0.8-2.5 um with up to 500 A astigmatism, 1/f^0.5 noise; one shared
    set of 1000 templates 180^2 from an 800-blob density in a 90-px ball;
    72 angles; window 512, overlap 200."""
    rng = np.random.default_rng(seed + 1000)
    sizes = [BATCH_SIZES[int(k)] for k in rng.integers(0, len(BATCH_SIZES), n_micrographs)]
    return dict(seed=seed, nx=sizes[0][0], ny=sizes[0][1], sizes=sizes, n_micrographs=n_micrographs,
                n_templates=1000, tsize=180, n_particles=250, snr=0.03, n_blobs=800, ball_radius=90.0,
                phistep=5.0, diameter=170.0, window=512, overlap=200, defocus=(0.8, 2.5),
                astig_A=500.0, noise_alpha=0.5, threshold=7.0, fast=True)


def config_full(seed: int = 1, window: int = 720) -> Dict[str, object]:
    """5760 x 4092 micrograph, 400 particles at SNR 0.03, 2000 templates 200^2
    from an 800-blob density in a 90-px ball, 72 angles, defocus 0.8-2.5 um
    with up to 500 A astigmatism, 1/f^0.5 coloured noise, window 720 with
    overlap 200."""
    return dict(seed=seed, nx=5760, ny=4092, n_templates=2000, tsize=200, n_particles=400,
                snr=0.03, n_blobs=800, ball_radius=90.0, phistep=5.0, diameter=190.0,
                window=window, overlap=200, defocus=(0.8, 2.5), astig_A=500.0,
                noise_alpha=0.5, threshold=7.0, fast=True)


def write_dataset(ds: Dataset, outdir: str, extra: Optional[Dict[str, object]] = None,
                  apix: float = 1.0) -> str:
    """Write MRCs, Euler file, list and config; returns the config path.

    All paths in the config and list are relative to ``outdir`` so that a run
    from ``outdir`` prints bare file names."""
    os.makedirs(outdir, exist_ok=True)
    formats.write_mrc(os.path.join(outdir, "templates.mrcs"), ds.templates, apix)
    formats.write_euler(os.path.join(outdir, "euler.lst"), ds.views)
    entries = []
    for m, mic in enumerate(ds.micrographs):
        name = "mic%03d.mrc" % m
        formats.write_mrc(os.path.join(outdir, name), mic.image, apix)
        entries.append((m, name, mic.defocus, mic.dfdiff, mic.dfang))
    formats.write_lst(os.path.join(outdir, "micrographs.lst"), entries)
    items = {"input": "micrographs.lst", "template": "templates.mrcs",
             "eulerfile": "euler.lst"}
    items.update(ds.params)
    items["output"] = "picks.lst"
    if extra:
        items.update(extra)
    path = os.path.join(outdir, "config")
    formats.write_config(path, items)
    return path
