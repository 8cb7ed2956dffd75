"""The oracle pinned against the reference's own kernels (CPU, no GPU).

oracle/_ref/libglsref.so is the reference's MetalPipeline/demosaic.metal
compiled as C++ against oracle/metal_shim and driven stage by stage by
oracle/ref_harness.cpp. Each test feeds both sides the same input (the
reference's output of the previous stage) and compares one stage:

  * the demosaic chain (interpolateGreen -> interpolateRedBlue ->
    interpolateRedBlueAtGreen -> blendHighlights) is FP32 in the reference
    too: the oracle's FP32 run must match it bit for bit;
  * the other stages compute in half precision in the reference
    (texture2d<half> kernels); the oracle's FP32 run must match them to a
    few half ulps (2^-11 relative; values are in [0, ~1.2]):
      scaleRawData, despeckles, quad branch: max |diff| <= 1e-3
      Sobel + gradient blur: 99.9% of pixels within 5e-4 (a pixel whose
        |blur(g)| < 4 sigma test flips after half rounding of the Sobel
        image takes the other blur);
      pyramid denoise (collectPatches, pcaProjection, block matching,
        reconstruct, in half): PSNR >= 70 dB, 99.9th pct <= 2e-3.
"""
import numpy as np
import pytest

import _oracle as O
import _ref as R
from glasscamerapublic_b200 import scene

pytestmark = pytest.mark.skipif(not R.available(), reason="reference kernels not built (make -C oracle ref)")


def _case(pattern=2, w=128, h=96, levels=3, iso=1600, seed=77, lsc=0.0):
    wl = scene.Workload("pin", w, h, levels=levels, gain=0.8, read=3.0, iso=iso, seed=seed, pattern=pattern)
    raw, clean = scene.make_raw(wl)
    p = scene.make_params(wl)
    p.lens_shading_correction = lsc
    return raw, p


def _stats(a, b):
    d = np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))
    return float(d.max()), float(np.quantile(d, 0.999))


@pytest.mark.parametrize("pattern", [0, 1, 2, 3])
@pytest.mark.parametrize("lsc", [0.0, 1.6])
def test_scale_raw_matches_reference_kernel(pattern, lsc):
    raw, p = _case(pattern, lsc=lsc)
    h, w = raw.shape
    ref = R.scale(raw, p)
    orc = O.stage("scale", p=p, w=w, h=h, out_shape=(h, w), raw=raw)
    mx, _ = _stats(ref, orc)
    assert mx <= 1e-3, mx


@pytest.mark.parametrize("pattern", [0, 1, 2, 3])
def test_demosaic_chain_is_bit_exact_to_reference_kernels(pattern):
    raw, p = _case(pattern)
    h, w = raw.shape
    s = R.scale(raw, p)
    g = R.sobel_blur(s, p)
    ref = R.demosaic_rgb(s, g, p)
    orc = O.stage("demosaic_rgb", s, g, p=p, w=w, h=h, out_shape=(h, w, 4))
    assert np.array_equal(ref[..., :3], orc[..., :3])
    # and with highlights above clip (blendHighlightsImage's branch)
    s2 = (s * (1.25 / np.quantile(s, 0.9))).astype(np.float32)  # top 10% above clip
    assert (s2 > 1).mean() > 0.05
    ref2 = R.demosaic_rgb(s2, g, p)
    orc2 = O.stage("demosaic_rgb", s2, g, p=p, w=w, h=h, out_shape=(h, w, 4))
    assert np.array_equal(ref2[..., :3], orc2[..., :3])


@pytest.mark.parametrize("pattern", [0, 2])
def test_sobel_blur_matches_reference_kernels(pattern):
    raw, p = _case(pattern)
    h, w = raw.shape
    s = R.scale(raw, p)
    ref = R.sobel_blur(s, p)
    orc = O.stage("sobel_blur", s, p=p, w=w, h=h, out_shape=(h, w, 2))
    _, q = _stats(ref, orc)
    assert q <= 5e-4, q


def test_high_noise_quad_branch_matches_reference_kernels():
    raw, p = _case(2, iso=1600)
    h, w = raw.shape
    s = R.scale(raw, p)
    g = R.sobel_blur(s, p)
    ref = R.raw_denoise(s, g, p)
    orc = O.stage("raw_denoise", s, g, p=p, w=w, h=h, out_shape=(h, w))
    mx, _ = _stats(ref, orc)
    assert mx <= 1e-3, mx


def test_despeckle_matches_reference_kernel():
    raw, p = _case(2)
    h, w = raw.shape
    s = R.scale(raw, p)
    g = R.sobel_blur(s, p)
    f, _ = O.cam_ycbcr(np.eye(3), scene.XYZ_SRGB)
    ycc = R.transform(R.demosaic_rgb(s, g, p), f)
    ref = R.despeckle(ycc, p)
    orc = O.stage("despeckle", ycc, p=p, w=w, h=h, out_shape=(h, w, 4))
    mx, _ = _stats(ref[..., :3], orc[..., :3])
    assert mx <= 1e-3, mx


@pytest.mark.parametrize("levels", [1, 3, 4])
def test_pyramid_denoise_matches_reference_kernels(levels):
    raw, p = _case(2, w=160, h=128, levels=levels)
    h, w = raw.shape
    s = R.scale(raw, p)
    g = R.sobel_blur(s, p)
    f, _ = O.cam_ycbcr(np.eye(3), scene.XYZ_SRGB)
    ycc = R.despeckle(R.transform(R.demosaic_rgb(s, g, p), f), p)
    ref, rbases = R.pyramid_denoise(ycc, g, p)
    orc = O.pyramid_denoise(ycc, g, p, f64=False)
    assert scene.psnr(ref[..., :3], orc["out"][..., :3]) >= 70.0
    _, q = _stats(ref[..., :3], orc["out"][..., :3])
    assert q <= 2e-3, q
    for l in range(levels):  # same PCA subspace
        a, b = rbases[l], orc["bases"][l]
        assert np.allclose(a @ a.T, b @ b.T, atol=1e-2), l


def test_full_chain_reference_kernels_vs_oracle():
    # the reference kernels end to end (host sequence of raw_converter.cpp)
    raw, p = _case(2, w=192, h=128, levels=4, iso=1600)
    h, w = raw.shape
    f, inv = O.cam_ycbcr(np.eye(3), scene.XYZ_SRGB)
    s = R.scale(raw, p)
    g = R.sobel_blur(s, p)
    if p.high_noise_image:
        s = R.raw_denoise(s, g, p)
    ycc = R.despeckle(R.transform(R.demosaic_rgb(s, g, p), f), p)
    den, _ = R.pyramid_denoise(ycc, g, p)
    ref = R.transform(den, inv)
    orc = O.raw_pipeline(raw, p, denoise=True, f64=False)["out"]
    assert scene.psnr(ref[..., :3], orc[..., :3]) >= 60.0


# ---------------------------------------------------------------- calibration
_ISOS = [1, 49, 50, 51, 99, 100, 150, 199, 200, 399, 400, 640, 800, 1000, 1599, 1600, 2500, 3200, 5000, 6399, 6400,
         6500, 10000, 12199, 12200, 12499, 12500, 20000]


def _fields(p):
    """The parameter fields a camera calibration fills, as float lists."""
    out = {"raw_a": list(p.raw_nlf.a), "raw_b": list(p.raw_nlf.b), "high_noise": p.high_noise_image,
           "raw_strength": p.raw_denoise_strength, "iso": p.iso, "lsc": p.lens_shading_correction,
           "rgb": [p.rgb_conversion.contrast, p.rgb_conversion.saturation, p.rgb_conversion.tone_curve_slope,
                   p.rgb_conversion.exposure_bias, p.rgb_conversion.blacks, p.rgb_conversion.local_tone_mapping],
           "ltm": [p.ltm.eps, p.ltm.shadows, p.ltm.highlights] + list(p.ltm.detail)}
    for l in range(5):
        out[f"nlf{l}"] = list(p.pyramid_nlf[l].a) + list(p.pyramid_nlf[l].b)
        d = p.denoise[l]
        out[f"den{l}"] = [d.luma, d.chroma, d.chroma_boost, d.gradient_boost, d.gradient_threshold, d.sharpening]
    return out


@pytest.mark.parametrize("iso", _ISOS)
def test_calibration_bit_exact_to_reference(native, iso):
    """gls_calibration_fill (the library's CameraCalibration) against the
    reference's own iPhone14WideCalibration compiled for the CPU
    (iPhone14WideCalibration.cpp:33-137, CameraCalibration.cpp:39-54):
    every field equal, including the integer-division ISO interpolation."""
    from glasscamerapublic_b200.api import iPhone14WideCalibration
    ours = _fields(iPhone14WideCalibration(levels=5).getDemosaicParameters(iso))
    ref = _fields(R.iPhone14WideCalibration(levels=5).getDemosaicParameters(iso))
    assert ours == ref, {k: (ours[k], ref[k]) for k in ours if ours[k] != ref[k]}
