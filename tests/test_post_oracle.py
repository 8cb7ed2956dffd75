"""The display post-processing (RawConverter::demosaic with postProcess) on
the CPU: the grain tables the library builds (gls_noise.h, through
gls_grain_tables) against the C library's srandom / random that the
reference calls, and known answers of the oracle's restatement
(oracle/gls_oracle_post.hpp): the histogram statistics, the tone curve and
the colour steps with tone mapping and grain off."""
import ctypes as C

import numpy as np
import pytest

import _oracle as O
import glasscamerapublic_b200 as g
from glasscamerapublic_b200 import scene


def _libc_random(seed, n):
    libc = C.CDLL(None)
    libc.random.restype = C.c_long
    libc.srandom.argtypes = [C.c_uint]
    libc.srandom(seed)
    return [libc.random() for _ in range(n)]


def _tables(seed):
    perm = np.zeros(514, np.int32)
    grad = np.zeros(1028, np.float32)
    g.check(g.lib().gls_grain_tables(seed, perm.ctypes.data_as(C.POINTER(C.c_int32)),
                                     grad.ctypes.data_as(C.POINTER(C.c_float))))
    return perm, grad.reshape(514, 2)


def _tables_from(rs):
    """Noise2D::initGradients (SimplexNoise.hpp:109-130) over a sequence of
    random() values."""
    it = iter(rs)
    perm = list(range(256))
    grad = np.zeros((514, 2), np.float32)
    for i in range(256):
        for j in range(2):
            grad[i, j] = np.float32((next(it) % 512) - 256) / np.float32(256)
        s = np.sqrt(np.float32(grad[i, 0] * grad[i, 0] + grad[i, 1] * grad[i, 1]), dtype=np.float32)
        grad[i] = grad[i] / s
    for i in range(255, 0, -1):
        k = perm[i]
        j = next(it) % 256
        perm[i] = perm[j]
        perm[j] = k
    perm = perm + [0] * 258
    for i in range(258):  # sequential, as the reference copies (the last two read the first copies)
        perm[256 + i] = perm[i]
        grad[256 + i] = grad[i]
    return np.array(perm, np.int32), grad


@pytest.mark.parametrize("seed", [1, 512, 4095, 65535])
def test_grain_tables_follow_the_c_library(seed):
    perm, grad = _tables(seed)
    rp, rg = _tables_from(_libc_random(seed, 512 + 255))
    assert np.array_equal(perm, rp)
    assert np.array_equal(grad, rg)
    assert sorted(perm[:256].tolist()) == list(range(256))


def _levels(w, h, seed=1):
    rng = np.random.default_rng(seed)
    return [rng.random((h >> l, w >> l, 4), dtype=np.float32) * 0.6 for l in range(5)]


def test_histogram_statistics_known_answers():
    w, h = 256, 192
    den = _levels(w, h)
    # level 3 (32 x 24) all at Y = 2 (255 / 255)^2 ... i.e. every count in bin 255
    den[3][..., 0] = 2.0
    p = scene.make_params(scene.Workload("pp", w, h, iso=800))
    rgb = np.zeros((h, w, 4), np.float32)
    grad = np.zeros((h, w, 2), np.float32)
    p.rgb_conversion.local_tone_mapping = 0
    _, st = O.postprocess(den, grad, rgb, p, 7)
    black, white, shadows, highlights, mean, median = st
    assert black == pytest.approx(2 * (254 / 255) ** 2)  # black index 255 -> v = 254/255
    assert white == pytest.approx(2.0)
    assert highlights == pytest.approx(3.0)  # all pixels in bands 5-7
    assert shadows == pytest.approx(0.8)
    assert median == pytest.approx(1.0 - black)
    assert mean == pytest.approx(1.0 - black)
    # a uniform Y = 0 image: every count in bin 0
    den[3][..., 0] = 0.0
    _, st = O.postprocess(den, grad, rgb, p, 7)
    assert st[0] == pytest.approx(2 * (1 / 255) ** 2)  # (0 - 1) / 255, squared
    assert st[2] == pytest.approx(0.3) and st[3] == pytest.approx(1.0)


def test_plain_colour_steps_without_tone_mapping_or_grain():
    w, h = 64, 48
    rng = np.random.default_rng(3)
    rgb = np.zeros((h, w, 4), np.float32)
    rgb[..., :3] = rng.random((h, w, 3), dtype=np.float32)
    grad = np.zeros((h, w, 2), np.float32)
    p = scene.make_params(scene.Workload("pp", w, h, iso=800))
    p.rgb_conversion.local_tone_mapping = 0
    p.rgb_conversion.contrast = 1.0
    p.rgb_conversion.saturation = 1.0
    for c in range(4):
        p.raw_nlf.a[c] = 0.0
        p.raw_nlf.b[c] = 0.0  # no grain
    out, st = O.postprocess(None, grad, rgb, p, 7, f64=True)  # without noise reduction: fixed levels
    assert st[0] == pytest.approx(0.1) and st[4] == pytest.approx(0.22)
    m = np.array(p.rgb_cam, np.float64).reshape(3, 3)
    pv = np.maximum(rgb[..., :3].astype(np.float64) - 0.1, 0) / 0.9
    x = np.maximum(pv @ m.T, 0)
    s = p.rgb_conversion.tone_curve_slope

    def sig(t):
        return 0.5 * (np.tanh(s * t - 0.3 * s) + 1)

    ref = np.clip((sig(np.sqrt(0.95 * x)) - sig(0.0)) / (sig(1.0) - sig(0.0)), 0, 1)
    assert np.abs(out[..., :3] - ref).max() < 1e-6
    assert np.all(out[..., 3] == 1)
