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


def step_chart(w: int, h: int, seed: int, cells: tuple = (12, 8)) -> np.ndarray:
    """A neutral step chart, (h, w, 3) float32: a grid of flat grey patches
    with levels spread over [0.01, 0.85] of white (log-spaced, shuffled),
    the kind of capture a noise model is measured on."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nx, ny = cells
    levels = np.geomspace(0.01, 0.85, nx * ny)
    rng.shuffle(levels)
    img = np.zeros((h, w, 3), dtype=np.float32)
    for j in range(ny):
        for i in range(nx):
            x0, x1 = i * w // nx, (i + 1) * w // nx
            y0, y1 = j * h // ny, (j + 1) * h // ny
            img[y0:y1, x0:x1, :] = levels[j * nx + i]
    return img


def make_chart_raw(wl: "Workload", frame: int = 0):
    """(raw uint16 (h, w), clean RGB) of a step chart at the workload's
    sensor noise."""
    seed = wl.seed + frame
    clean = step_chart(wl.width, wl.height, seed)
    raw = add_noise(mosaic(clean, wl.pattern), wl.black, wl.white, wl.gain, wl.read, seed)
    return raw, clean


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
    "cfg3_burst_4032x3024": Workload("cfg3_burst_4032x3024", 4032, 3024, levels=5, gain=1.5, read=4.0, iso=800,
                                     seed=3000, extra={"frames": 8}),
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


def burst_homographies(n: int, w: int, h: int, seed: int, max_rot_deg: float = 1.0, max_shift: float = 20.0,
                       max_persp: float = 1e-5) -> list:
    """Frame i's homography H_i (3x3 float64) mapping reference-frame pixels
    to frame-i pixels, p_i ~ H_i p_ref; frame 0 is the reference (identity).
    Rotation about the image centre within +-max_rot_deg, shift within
    +-max_shift px, perspective terms within +-max_persp."""
    rng = np.random.Generator(np.random.PCG64(seed ^ 0xB0B))
    out = [np.eye(3)]
    cx, cy = (w - 1) / 2.0, (h - 1) / 2.0
    for _ in range(1, n):
        a = np.deg2rad(rng.uniform(-max_rot_deg, max_rot_deg))
        tx, ty = rng.uniform(-max_shift, max_shift, size=2)
        px, py = rng.uniform(-max_persp, max_persp, size=2)
        c, s_ = np.cos(a), np.sin(a)
        T0 = np.array([[1, 0, -cx], [0, 1, -cy], [0, 0, 1.0]])
        R = np.array([[c, -s_, 0], [s_, c, 0], [0, 0, 1.0]])
        T1 = np.array([[1, 0, cx + tx], [0, 1, cy + ty], [0, 0, 1.0]])
        P = np.array([[1, 0, 0], [0, 1, 0], [px, py, 1.0]])
        H = T1 @ R @ T0 @ P
        out.append(H / H[2, 2])
    return out


def warp_rgb(img: np.ndarray, H_ref_to_frame: np.ndarray) -> np.ndarray:
    """Frame = reference image seen through H: frame(x) = ref(H^-1 x),
    bilinear, clamp-to-edge."""
    h, w = img.shape[:2]
    Hi = np.linalg.inv(H_ref_to_frame)
    ys, xs = np.mgrid[0:h, 0:w].astype(np.float64)
    den = Hi[2, 0] * xs + Hi[2, 1] * ys + Hi[2, 2]
    u = np.clip((Hi[0, 0] * xs + Hi[0, 1] * ys + Hi[0, 2]) / den, 0, w - 1)
    v = np.clip((Hi[1, 0] * xs + Hi[1, 1] * ys + Hi[1, 2]) / den, 0, h - 1)
    x0 = np.minimum(np.floor(u).astype(np.int64), w - 2)
    y0 = np.minimum(np.floor(v).astype(np.int64), h - 2)
    fx = (u - x0)[..., None]
    fy = (v - y0)[..., None]
    a = img[y0, x0] * (1 - fx) + img[y0, x0 + 1] * fx
    b = img[y0 + 1, x0] * (1 - fx) + img[y0 + 1, x0 + 1] * fx
    return (a * (1 - fy) + b * fy).astype(np.float32)


def textured_scene(w: int, h: int, seed: int, blobs_per_mpx: float = 400.0) -> np.ndarray:
    """clean_scene plus small square and round blobs (2 to 24 px across,
    about blobs_per_mpx per megapixel): the local structure a feature
    detector registers on."""
    img = clean_scene(w, h, seed).astype(np.float64)
    rng = np.random.Generator(np.random.PCG64(seed ^ 0xB10B))
    n = int(blobs_per_mpx * w * h / 1e6)
    mean = img.mean()
    for _ in range(n):
        r = rng.uniform(1.0, 12.0)
        cx, cy = rng.uniform(0, w), rng.uniform(0, h)
        x0, x1 = int(max(cx - r, 0)), int(min(cx + r + 1, w))
        y0, y1 = int(max(cy - r, 0)), int(min(cy + r + 1, h))
        if x1 <= x0 or y1 <= y0:
            continue
        col = rng.uniform(0.2, 3.0, size=3) * mean
        if rng.uniform() < 0.5:
            yy, xx = np.mgrid[y0:y1, x0:x1]
            m = (xx - cx) ** 2 + (yy - cy) ** 2 <= r * r
            img[y0:y1, x0:x1][m] = col
        else:
            img[y0:y1, x0:x1] = col
    return np.clip(img, 0.0, 1.0).astype(np.float32)


def make_burst(wl: Workload, n: int | None = None):
    """A burst of n raw frames of one textured scene, frame i warped by H_i
    (burst_homographies): (raws, cleans, homographies)."""
    n = n or int(wl.extra.get("frames", 8))
    ref = textured_scene(wl.width, wl.height, wl.seed)
    Hs = burst_homographies(n, wl.width, wl.height, wl.seed)
    raws, cleans = [], []
    for i, H in enumerate(Hs):
        c = ref if i == 0 else warp_rgb(ref, H)
        cleans.append(c)
        raws.append(add_noise(mosaic(c, wl.pattern), wl.black, wl.white, wl.gain, wl.read, wl.seed + i))
    return raws, cleans, Hs


def corner_error(H_est, H_true, w: int, h: int) -> float:
    """Largest distance (px) between the image corners mapped by the two
    homographies."""
    pts = np.array([[0, 0, 1], [w - 1, 0, 1], [0, h - 1, 1], [w - 1, h - 1, 1]], np.float64).T
    a = np.asarray(H_est, np.float64) @ pts
    b = np.asarray(H_true, np.float64) @ pts
    return float(np.max(np.hypot(a[0] / a[2] - b[0] / b[2], a[1] / a[2] - b[1] / b[2])))


def target_rgb(clean: np.ndarray) -> np.ndarray:
    """The noise-free output the pipeline aims at, in its scaled units
    (0.1 + 0.9 * linear, identity camera matrix)."""
    return 0.1 + 0.9 * clean


def psnr(a: np.ndarray, b: np.ndarray, peak: float = 1.0) -> float:
    mse = float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))
    return float("inf") if mse == 0 else 10.0 * math.log10(peak * peak / mse)
