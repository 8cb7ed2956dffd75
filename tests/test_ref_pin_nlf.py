"""The oracle's noise-model measurement (calibrateFromImage,
oracle/gls_oracle_nlf.hpp) pinned against the reference's own code compiled
for the CPU (no GPU):

  * basicRawNoiseStatistics / basicNoiseStatistics (demosaic.metal:1110-1159),
    the reference's kernels through oracle/metal_shim: bit-exact;
  * RawConverter::MeasureRawNLF (raw_converter.cpp:339-490) and
    PyramidProcessor::MeasureYCbCrNLF (pyramid_processor.cpp:173-324), the
    reference's own host code (oracle/ref_nlf.cpp over oracle/gls_shim/
    gls_nlf.hpp): the measured models are bit-exact (float results of the
    same FP64 sums in the same order).

Inputs are neutral step charts (the captures a noise model is measured on)
and the synthetic natural scene, whose edges make the second fit fail its
acceptance test, so both branches of the reference's two-pass fit run.
"""
import numpy as np
import pytest

import _oracle as O
import _ref as R
from glasscamerapublic_b200 import scene

pytestmark = pytest.mark.skipif(not R.available(), reason="reference kernels not built (make -C oracle ref)")

SENSORS = [(100, 2.0, 2.0), (1600, 0.5, 4.0), (6400, 0.15, 6.0)]


def _frame(w=512, h=384, iso=1600, gain=0.5, read=4.0, seed=3, pattern=2, chart=True):
    wl = scene.Workload("nlf", w, h, levels=5, gain=gain, read=read, iso=iso, seed=seed, pattern=pattern)
    raw, _ = (scene.make_chart_raw if chart else scene.make_raw)(wl)
    return raw, scene.make_params(wl)


@pytest.mark.parametrize("pattern", [0, 1, 2, 3])
@pytest.mark.parametrize("w,h", [(256, 192), (130, 98)])
def test_raw_statistics_are_the_reference_kernel(pattern, w, h):
    raw, p = _frame(w, h, pattern=pattern, chart=False)
    s = R.scale(raw, p)
    rm, rv = R.raw_noise_stats(s, pattern)
    om, ov = O.raw_noise_stats(s, pattern)
    assert np.array_equal(rm, om) and np.array_equal(rv, ov)


@pytest.mark.parametrize("iso,gain,read", SENSORS)
@pytest.mark.parametrize("chart", [True, False])
def test_measure_raw_nlf_is_the_reference_regression(iso, gain, read, chart):
    raw, p = _frame(iso=iso, gain=gain, read=read, chart=chart)
    h, w = raw.shape
    mean, var = R.raw_noise_stats(R.scale(raw, p), p.bayer_pattern)
    for exposure in (1.0, 1.7):
        ra, rb = R.measure_raw_nlf(mean, var, w, h, exposure)
        oa, ob = O.measure_raw_nlf(mean, var, w, h, exposure)
        assert np.array_equal(ra, oa) and np.array_equal(rb, ob), (ra, oa, rb, ob)


def test_measured_raw_slope_on_a_step_chart_is_the_sensor_model():
    # variance = a + b y with b = 0.9 / (gain (white - black)): the fit over
    # the flat patches recovers b to within the patch edges' bias
    for iso, gain, read in SENSORS:
        raw, p = _frame(iso=iso, gain=gain, read=read)
        h, w = raw.shape
        mean, var = O.raw_noise_stats(O.stage("scale", p=p, w=w, h=h, out_shape=(h, w), raw=raw), p.bayer_pattern)
        a, b = O.measure_raw_nlf(mean, var, w, h)
        true_b = p.raw_nlf.b[1]
        assert np.all(np.abs(b / true_b - 1) < 0.1), (b, true_b)


def _levels(img, n=5):
    out = [np.ascontiguousarray(img, np.float32)]
    for i in range(1, n):
        h, w = out[-1].shape[:2]
        out.append(O.downsample(out[-1], w // 2, h // 2, f64=False))
    return out


@pytest.mark.parametrize("iso,gain,read", SENSORS)
@pytest.mark.parametrize("chart", [True, False])
def test_ycbcr_statistics_and_fit_are_the_reference(iso, gain, read, chart):
    raw, p = _frame(iso=iso, gain=gain, read=read, chart=chart)
    ds = O.raw_pipeline(raw, p, denoise=True, f64=False, stages=True)["despeckled"]
    for lvl in _levels(ds):
        rs = R.ycc_noise_stats(lvl)
        os_ = O.ycc_noise_stats(lvl)
        assert np.array_equal(rs, os_)
        for exposure in (1.0, 0.6):
            ra, rb = R.measure_ycc_nlf(rs, exposure)
            oa, ob = O.measure_ycc_nlf(os_, exposure)
            assert np.array_equal(ra, oa) and np.array_equal(rb, ob), (lvl.shape, ra, oa, rb, ob)


def test_flat_frame_has_no_variance_class():
    # a constant frame at 0.58: rounding leaves every variance negative
    # (-1.04e-6); the reference then indexes its histogram with an undefined
    # value; the oracle leaves such positions out of the histogram (so the
    # variance bound stays 1) and the degenerate fit stays finite and floored
    w, h = 64, 48
    s = np.full((h, w), 0.58, np.float32)
    mean, var = O.raw_noise_stats(s, 2)
    assert (var[..., 0] < 0).all()
    a, b = O.measure_raw_nlf(mean, var, w, h)
    assert np.all(np.isfinite(a)) and np.all(a >= np.float32(1e-8)) and np.all(b >= np.float32(1e-8))
    assert R.lib().ref_measure_raw_nlf(R._fp(mean), R._fp(var), w, h, 1.0, R._fp(a), R._fp(b)) == 2


def test_calibrated_pipeline_uses_the_measured_models():
    raw, p = _frame(w=384, h=256, iso=1600, gain=0.5, read=4.0)
    out, (ra, rb), pyr = O.raw_pipeline_calibrated(raw, p)
    h, w = raw.shape
    s = O.stage("scale", p=p, w=w, h=h, out_shape=(h, w), raw=raw)
    mean, var = O.raw_noise_stats(s, p.bayer_pattern)
    a, b = O.measure_raw_nlf(mean, var, w, h)
    assert np.array_equal(a, ra) and np.array_equal(b, rb)
    # the front end with the measured raw model and the high-noise branch
    # off; despeckling with the given level-0 model; each level measured
    q = type(p).from_buffer_copy(p)
    q.high_noise_image = 0
    for c in range(4):
        q.raw_nlf.a[c], q.raw_nlf.b[c] = float(ra[c]), float(rb[c])
    ds = O.raw_pipeline(raw, q, denoise=True, f64=False, stages=True)["despeckled"]
    for l, lvl in enumerate(_levels(ds, p.levels)):
        la, lb = O.measure_ycc_nlf(O.ycc_noise_stats(lvl))
        assert np.array_equal(la, pyr[l, 0]) and np.array_equal(lb, pyr[l, 1]), l
    # and the denoise runs on the measured models
    for l in range(p.levels):
        for c in range(3):
            q.pyramid_nlf[l].a[c], q.pyramid_nlf[l].b[c] = float(pyr[l, 0, c]), float(pyr[l, 1, c])
    den = O.pyramid_denoise(ds, O.raw_pipeline(raw, q, denoise=False, f64=False, stages=True)["gradient"], q,
                            f64=False)["out"]
    f, inv = O.cam_ycbcr(np.array(p.rgb_cam, np.float64).reshape(3, 3), np.array(p.xyz_rgb, np.float64).reshape(3, 3))
    rgb = den[..., :3] @ np.asarray(inv, np.float64).reshape(3, 3).T
    assert np.abs(rgb - out[..., :3]).max() < 1e-5
