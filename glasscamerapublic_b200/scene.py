"""Seeded synthetic raw scenes and parameter blocks for the workloads.

The reference measures on DNG bursts that are not available here; these
scenes stand in for them with the shapes, bit depths and noise levels of the
five workloads:

  * a 3-octave gradient-noise RGB field (Perlin-style lattice gradients,
    persistence 0.5), scaled so the mean signal is 18% of white,
  * 20 axis-aligned hard-edged rectangles of random colours (a few near
    clipping, to exercise the highlight blend),
  * Poisson-Gaussian noise: Poisson(electrons = DN * gain) / gain +
    N(0, read^2) + black, rounded and clipped to [0, white],
  * sampled to a Bayer mosaic with the kernels' channel offsets.

Everything is generated by numpy's PCG64 from an explicit seed, so every
run (CPU oracle and GPU) sees identical bytes.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import RGGB, DemosaicParams

# Bayer offsets (x, y) of R, G, B, G2 per pattern (demosaic.metal:33-38)
BAYER_OFFSETS = {
    0: ((1, 0), (0, 0), (0, 1), (1, 1)),
    1: ((0, 1), (0, 0), (1, 0), (1, 1)),
    2: ((0, 0), (0, 1), (1, 1), (1, 0)),
    3: ((1, 1), (0, 1), (0, 0), (1, 0)),
}

XYZ_SRGB = (0.4124, 0.3576, 0.1805, 0.2126, 0.7152, 0.0722, 0.0193, 0.1192, 0.9505)


def _fade(t):
    return t * t * t * (t * (t * 6 - 15) + 10)


def gradient_noise(w: int, h: int, period: float, rng: np.random.Generator) -> np.ndarray:
    """One octave of lattice gradient noise in [-1, 1] (approximately)."""
    gw, gh = int(math.ceil(w / period)) + 2, int(math.ceil(h / period)) + 2
    ang = rng.uniform(0, 2 * np.pi, size=(gh, gw))
    gx, gy = np.cos(ang), np.sin(ang)
    xs = np.arange(w, dtype=np.float64) / period
    ys = np.arange(h, dtype=np.float64) / period
    x0 = np.floor(xs).astype(np.int64)
    y0 = np.floor(ys).astype(np.int64)
    fx = (xs - x0)[None, :]
    fy = (ys - y0)[:, None]
    X0, Y0 = x0[None, :], y0[:, None]

    def dot(ix, iy, dx, dy):
        return gx[iy, ix] * dx + gy[iy, ix] * dy

    n00 = dot(X0, Y0, fx, fy)
    n10 = dot(X0 + 1, Y0, fx - 1, fy)
    n01 = dot(X0, Y0 + 1, fx, fy - 1)
    n11 = dot(X0 + 1, Y0 + 1, fx - 1, fy - 1)
    u, v = _fade(fx), _fade(fy)
    top = n00 + (n10 - n00) * u
    bot = n01 + (n11 - n01) * u
    return (top + (bot - top) * v) * 1.4142


def clean_scene(w: int, h: int, seed: int, n_rect: int = 20) -> np.ndarray:
    """Linear RGB scene in [0, 1] relative to white - black, (h, w, 3) float32."""
    rng = np.random.Generator(np.random.PCG64(seed))
    img = np.zeros((h, w, 3), dtype=np.float64)
    base = max(w, h) / 6.0
    for c in range(3):
        acc = np.zeros((h, w))
        amp, per = 1.0, base
        for _ in range(3):
            acc += amp * gradient_noise(w, h, per, rng)
            amp *= 0.5
            per *= 0.5
        img[..., c] = 0.5 + 0.35 * acc
    img = np.clip(img, 0.0, 1.0)
    for _ in range(n_rect):
        rw = int(rng.uniform(w / 20, w / 4))
        rh = int(rng.uniform(h / 20, h / 4))
        x = int(rng.uniform(0, max(1, w - rw)))
        y = int(rng.uniform(0, max(1, h - rh)))
        col = rng.uniform(0.02, 0.9, size=3)
        if rng.uniform() < 0.15:
            col = rng.uniform(0.9, 1.0, size=3)
        img[y:y + rh, x:x + rw, :] = col
    # mean signal at 18% of white
    img *= 0.18 / img.mean()
    return np.clip(img, 0.0, 1.0).astype(np.float32)


def mosaic(rgb: np.ndarray, pattern: int = RGGB) -> np.ndarray:
    """Sample a linear RGB image to a Bayer mosaic (float, same units)."""
    h, w = rgb.shape[:2]
    out = np.empty((h, w), dtype=rgb.dtype)
    chan = (0, 1, 2, 1)  # R, G, B, G2 -> RGB channel
    for c, (ox, oy) in enumerate(BAYER_OFFSETS[pattern]):
        out[oy::2, ox::2] = rgb[oy::2, ox::2, chan[c]]
    return out


def add_noise(m: np.ndarray, black: int, white: int, gain: float, read: float, seed: int) -> np.ndarray:
    """Poisson-Gaussian sensor noise; returns uint16 raw DN."""
    rng = np.random.Generator(np.random.PCG64(seed ^ 0x5EED))
    dn = m.astype(np.float64) * (white - black)
    e = rng.poisson(np.maximum(dn * gain, 0.0))
    noisy = e / gain + rng.normal(0.0, read, size=m.shape) + black
    return np.clip(np.rint(noisy), 0, white).astype(np.uint16)


def raw_nlf(black: int, white: int, gain: float, read: float):
    """Analytic raw NLF in scaled units y = 0.9 (DN - black)/(white - black) + 0.1:
    var(y) = a + b y with b = 0.9 / (g (white - black)),
    a = 0.81 r^2 / (white - black)^2 - 0.1 b (floored at 1e-8)."""
    rng_ = white - black
    b = 0.9 / (gain * rng_)
    a = max(0.81 * read * read / (rng_ * rng_) - 0.1 * b, 1e-8)
    return a, b


@dataclass
class Workload:
    name: str
    width: int
    height: int
    levels: int = 5
    black: int = 512
    white: int = 4095
    gain: float = 2.0
    read: float = 5.0
    iso: int = 1600
    pattern: int = RGGB
    seed: int = 0
    extra: dict = field(default_factory=dict)


# the five reference workloads (sizes, bit depths and noise of each)
WORKLOADS = {
    "cfg1_1024x768": Workload("cfg1_1024x768", 1024, 768, levels=4, gain=0.8, read=3.0, iso=200, seed=1000),
    "cfg2_4032x3024": Workload("cfg2_4032x3024", 4032, 3024, levels=5, gain=2.0, read=5.0, iso=1600, seed=2000),
}

MIXED_SIZES = [(4032, 3024), (6000, 4000), (5472, 3648), (8368, 5584)]


def mixed_batch(n_each: int = 4):
    """The 16-frame mixed-sensor batch: sizes, 12/14-bit whites, per-frame noise."""
    out = []
    rng = np.random.Generator(np.random.PCG64(4000))
    k = 0
    for (w, h) in MIXED_SIZES:
        for i in range(n_each):
            white = 4095 if (k % 2 == 0) else 16383
            black = 512 if white == 4095 else 2048
            gain = float(rng.uniform(0.5, 3.0))
            read = float(rng.uniform(2.0, 6.0))
            out.append(Workload(f"cfg4_{w}x{h}_{i}", w, h, levels=5, black=black, white=white, gain=gain,
                                read=read, iso=800, seed=4000 + k))
            k += 1
    return out


def make_params(wl: Workload, calibration=None) -> DemosaicParams:
    """DemosaicParameters of a workload: identity camera matrix, sRGB primaries,
    scale_mul = 65535 / (white - black), analytic raw NLF, pyramid NLF and
    denoise schedule from the camera calibration at the workload's ISO."""
    from .api import iPhone14WideCalibration
    cal = calibration or iPhone14WideCalibration(levels=wl.levels)
    p = cal.getDemosaicParameters(wl.iso)
    p.bayer_pattern = wl.pattern
    p.black_level = float(wl.black)
    p.white_level = float(wl.white)
    p.exposure_multiplier = 1.0
    p.lens_shading_correction = 0.0
    for c in range(4):
        p.scale_mul[c] = 65535.0 / (wl.white - wl.black)
    for i in range(9):
        p.rgb_cam[i] = 1.0 if i in (0, 4, 8) else 0.0
        p.xyz_rgb[i] = XYZ_SRGB[i]
    a, b = raw_nlf(wl.black, wl.white, wl.gain, wl.read)
    for c in range(4):
        p.raw_nlf.a[c] = a
        p.raw_nlf.b[c] = b
    p.levels = wl.levels
    return p


def make_raw(wl: Workload, frame: int = 0):
    """(raw uint16 (h, w), clean linear RGB (h, w, 3)) of a workload frame."""
    seed = wl.seed + frame
    clean = clean_scene(wl.width, wl.height, seed)
    raw = add_noise(mosaic(clean, wl.pattern), wl.black, wl.white, wl.gain, wl.read, seed)
    return raw, clean


def target_rgb(clean: np.ndarray) -> np.ndarray:
    """The noise-free output the pipeline aims at, in its scaled units
    (0.1 + 0.9 * linear, identity camera matrix)."""
    return 0.1 + 0.9 * clean


def psnr(a: np.ndarray, b: np.ndarray, peak: float = 1.0) -> float:
    mse = float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))
    return float("inf") if mse == 0 else 10.0 * math.log10(peak * peak / mse)
