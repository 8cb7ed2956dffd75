"""The oracle's display post-processing (oracle/gls_oracle_post.hpp) pinned
against the reference's own kernels (CPU, no GPU).

oracle/_ref/libglsref.so runs MetalPipeline/demosaic.metal:1292-1723
(GuidedFilterABImage, BoxFilterGFImage, histogramImage,
histogramStatistics, localToneMappingMaskImage, convertTosRGB) as C++
against oracle/metal_shim in the host order of raw_converter.cpp, with the
grain tables of the reference's own Noise2D (SimplexNoise.hpp). Both sides
take the same inputs: five denoised levels, the level-0 gradient and the
linear camera RGB of a scene run through the oracle's raw path.

These kernels compute in FP32 in the reference (texture2d<float>) and the
oracle's FP32 run follows their operation order, so:
  * the grain tables and the histogram statistics are bit-exact;
  * for power-of-two frame sizes the picture is bit-exact too;
  * for other sizes the reference's normalised sampler coordinates
    (pos + (offset + 0.5) / size, then * size - 0.5 in the sampler) carry
    float rounding that the oracle's integer texel offsets do not (a Metal
    sampler snaps such sub-ulp offsets away with its fixed-point weights);
    the picture then matches to max |diff| <= 5e-5.
"""
import ctypes as C

import numpy as np
import pytest

import _oracle as O
import _ref as R
import glasscamerapublic_b200 as g
from glasscamerapublic_b200 import scene

pytestmark = pytest.mark.skipif(not R.available(), reason="reference kernels not built (make -C oracle ref)")


def _inputs(w=256, h=256, iso=1600, seed=41, pattern=2):
    wl = scene.Workload("pin-post", w, h, levels=5, gain=0.8, read=3.0, iso=iso, seed=seed, pattern=pattern)
    raw, clean = scene.make_raw(wl)
    p = scene.make_params(wl)
    st = O.raw_pipeline(raw, p, denoise=True, f64=False, stages=True)
    den = O.pyramid_denoise(st["despeckled"], st["gradient"], p, f64=False, levels_out=True)["levels"]
    return raw, p, den, st["gradient"], st["out"]


_CASE = {}


@pytest.fixture
def case():
    """256 x 256 inputs, built once; a fresh copy of the parameters per test."""
    if not _CASE:
        _CASE["v"] = _inputs()
    raw, p, den, grad, rgb = _CASE["v"]
    return raw, type(p).from_buffer_copy(p), den, grad, rgb


@pytest.mark.parametrize("seed", [0, 1, 77, 4095])
def test_grain_tables_are_the_reference_noise2d(seed):
    rp, rg = R.noise_tables(seed)
    perm = np.zeros(514, np.int32)
    grad = np.zeros((514, 2), np.float32)
    g.check(g.lib().gls_grain_tables(seed, perm.ctypes.data_as(C.POINTER(C.c_int32)),
                                     grad.ctypes.data_as(C.POINTER(C.c_float))))
    assert np.array_equal(perm, rp)
    assert np.array_equal(grad, rg)


def _compare(den, grad, rgb, p, seed, tol=0.0):
    ref, rst = R.postprocess(den, grad, rgb, p, seed)
    orc, ost = O.postprocess(den, grad, rgb, p, seed)
    assert np.array_equal(rst, ost), (rst, ost)
    d = np.abs(ref.astype(np.float64) - orc)
    assert d.max() <= tol, (float(d.max()), np.unravel_index(int(d.argmax()), d.shape))
    return ref, rst


def test_default_post_processing_matches_reference_kernels(case):
    raw, p, den, grad, rgb = case
    ref, st = _compare(den, grad, rgb, p, int(raw[0, 0]))
    assert np.all(ref[..., 3] == 1) and ref[..., :3].min() >= 0 and ref[..., :3].max() <= 1
    assert 0 < st[2] <= 0.8 and 1 <= st[3] <= 3  # shadows, highlights in their ranges


@pytest.mark.parametrize("contrast,saturation,bias,blacks", [(1.0, 1.0, 0.0, 0.0), (1.3, 1.4, 0.7, 0.02),
                                                              (0.8, 0.6, -0.5, 0.0)])
def test_colour_controls_match_reference_kernels(case, contrast, saturation, bias, blacks):
    raw, p, den, grad, rgb = case
    rc = p.rgb_conversion
    rc.contrast, rc.saturation, rc.exposure_bias, rc.blacks = contrast, saturation, bias, blacks
    _compare(den, grad, rgb, p, 123)


@pytest.mark.parametrize("detail", [(1.0, 1.0, 1.0), (1.0, 1.5, 2.0), (2.0, 1.2, 3.0), (0.8, 0.9, 1.0)])
@pytest.mark.parametrize("eps", [0.01, 0.001])
def test_tone_mapping_mask_matches_reference_kernels(case, detail, eps):
    raw, p, den, grad, rgb = case
    p.ltm.eps = eps
    for k in range(3):
        p.ltm.detail[k] = detail[k]
    _compare(den, grad, rgb, p, 5)


def test_without_tone_mapping_and_without_grain(case):
    raw, p, den, grad, rgb = case
    p.rgb_conversion.local_tone_mapping = 0
    _compare(den, grad, rgb, p, 9)
    for c in range(4):
        p.raw_nlf.a[c] = 0.0
        p.raw_nlf.b[c] = 0.0
    _compare(den, grad, rgb, p, 9)


def test_without_noise_reduction_uses_fixed_statistics(case):
    raw, p, den, grad, rgb = case
    p.rgb_conversion.local_tone_mapping = 0  # the reference computes no mask without noise reduction
    ref, st = _compare(None, grad, rgb, p, 17)
    assert st[0] == pytest.approx(0.1) and st[4] == pytest.approx(0.22) and st[5] == pytest.approx(0.22)


def test_histogram_extremes_match_reference_kernels(case):
    raw, p, den, grad, rgb = case
    d = [x.copy() for x in den]
    d[3][..., 0] = 0.0  # every count in bin 0
    _compare(d, grad, rgb, p, 3)
    d[3][..., 0] = 5.0  # every count clamped into bin 255
    _compare(d, grad, rgb, p, 3)
    d[3][..., 0] = np.linspace(0, 2, d[3].shape[1], dtype=np.float32)[None, :]  # a ramp over all bins
    _compare(d, grad, rgb, p, 3)


@pytest.mark.parametrize("w,h", [(256, 192), (200, 136), (328, 216)])
def test_other_frame_sizes(w, h):
    raw, p, den, grad, rgb = _inputs(w=w, h=h, seed=43)
    _compare(den, grad, rgb, p, int(raw[0, 0]), tol=5e-5)
    p.rgb_conversion.local_tone_mapping = 0  # no sampler: bit-exact again
    _compare(den, grad, rgb, p, int(raw[0, 0]))


@pytest.mark.parametrize("w,h,iso", [(256, 256, 1600), (320, 240, 200)])
def test_end_to_end_with_post_processing_vs_reference_kernels(w, h, iso):
    # RawConverter::demosaic(postProcess=true) through the reference kernels
    # (half-precision pyramid) against the oracle's FP32 chain
    raw, p, den, grad, rgb = _inputs(w=w, h=h, iso=iso)
    orc, ost = O.postprocess(den, grad, rgb, p, int(raw[0, 0]))
    ref, rst = R.demosaic_post(raw, p)
    assert scene.psnr(orc[..., :3], ref[..., :3]) >= 58.0
    assert np.allclose(ost, rst, atol=2e-4)  # counts move only where the half-precision levels differ
