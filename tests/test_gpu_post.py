"""GPU parity of the display post-processing (GLS_POSTPROCESS,
RawConverter::demosaic with postProcess, raw_converter.cpp:226-242) against
the oracle's restatement (oracle/gls_oracle_post.hpp), through the C ABI.

The oracle is fed the CUDA path's own intermediate planes of the same call
(the five denoised levels, the level-0 gradient and the linear camera RGB of
a run without post-processing), with the grain seeded from the raw frame's
first pixel, so the comparison isolates the post-processing kernels.

Tolerances (outputs in [0, 1]; FP32 and FP16 storage alike, the oracle fed
the planes the path stored): 99.9th percentile of |diff| <= 5e-6, max
<= 2e-4. Measured on B200: 99.9th percentiles of 2-5e-7 and maxima of
1e-6 to 2e-5 (1024 x 768). The kernels' pow is exp2(y log2 x) and their
sigmoid a logistic of exp2, a few ulps from the oracle's C library calls,
which the tone-mapping powers amplify near dark pixels.
"""
import numpy as np
import pytest

import _oracle as O
import _ref as R
import glasscamerapublic_b200 as g
from glasscamerapublic_b200 import scene

pytestmark = pytest.mark.gpu


def _frame(w=256, h=192, iso=800, seed=5):
    wl = scene.Workload("pp", w, h, levels=5, gain=0.8, read=3.0, iso=iso, seed=seed)
    raw, clean = scene.make_raw(wl)
    return raw, scene.make_params(wl)


def _p999(a, b):
    d = np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))
    return float(np.quantile(d, 0.999)), float(d.max())


def _planes(conv, levels=5):
    den = [conv.plane(g.PLANE_DENOISED_L0 + l).astype(np.float32) for l in range(levels)]
    return den, conv.plane(g.PLANE_GRADIENT).astype(np.float32)


def _post_vs_oracle(conv, raw, p, fp16=False, denoise=True):
    out = conv.demosaic(raw, p, noiseReduction=denoise, fp16=fp16, postProcess=True)
    den, grad = _planes(conv) if denoise else (None, conv.plane(g.PLANE_GRADIENT).astype(np.float32))
    rgb = conv.demosaic(raw, p, noiseReduction=denoise, fp16=fp16).astype(np.float32)
    ref, stats = O.postprocess(den, grad, rgb, p, int(raw[0, 0]))
    return out, ref, stats


@pytest.mark.parametrize("ltm", [1, 0])
def test_post_fp32_matches_oracle(converter, ltm):
    raw, p = _frame()
    p.rgb_conversion.local_tone_mapping = ltm
    out, ref, _ = _post_vs_oracle(converter, raw, p)
    q, m = _p999(out, ref)
    assert q <= 5e-6 and m <= 2e-4, (q, m)
    assert np.all(out[..., 3] == 1)
    assert out[..., :3].min() >= 0 and out[..., :3].max() <= 1


def test_post_without_noise_reduction(converter):
    raw, p = _frame(seed=9)
    out, ref, stats = _post_vs_oracle(converter, raw, p, denoise=False)
    q, m = _p999(out, ref)
    assert q <= 5e-6 and m <= 2e-4, (q, m)
    assert stats[0] == pytest.approx(0.1) and stats[4] == pytest.approx(0.22)


@pytest.mark.parametrize("w,h,iso", [(512, 384, 3200), (320, 208, 100)])
def test_post_fp16_storage_matches_oracle(converter, w, h, iso):
    raw, p = _frame(w, h, iso=iso, seed=11)
    out, ref, _ = _post_vs_oracle(converter, raw, p, fp16=True)
    q, m = _p999(out, ref)
    assert q <= 5e-6 and m <= 2e-4, (q, m)


def test_grain_follows_the_first_raw_pixel(converter):
    raw, p = _frame(seed=13)
    a = converter.demosaic(raw, p, postProcess=True)
    raw2 = raw.copy()
    raw2[0, 0] = raw[0, 0] + 1  # a new grain seed; the pixel itself hardly moves the picture
    b = converter.demosaic(raw2, p, postProcess=True)
    den, grad = _planes(converter)
    rgb = converter.demosaic(raw2, p).astype(np.float32)
    ref, _ = O.postprocess(den, grad, rgb, p, int(raw2[0, 0]))
    q, m = _p999(b, ref)
    assert q <= 5e-6 and m <= 2e-4, (q, m)
    assert np.abs(a - b)[8:, 8:].max() > 1e-4  # the grain moved


def test_post_batch_matches_single_frames(converter):
    import torch
    frames = [_frame(256, 192, iso=800, seed=21), _frame(320, 240, iso=1600, seed=22)]
    outs, singles = [], []
    for raw, p in frames:
        singles.append(converter.demosaic(raw, p, fp16=True, postProcess=True))
        outs.append(torch.empty((raw.shape[0], raw.shape[1], 4), dtype=torch.float32, device="cuda"))
    draws = [torch.from_numpy(r.view(np.int16)).cuda() for r, _ in frames]
    converter.demosaic_batch(draws, [p for _, p in frames], outs, fp16=True, out_fp16=False, sync=True,
                             postProcess=True)
    torch.cuda.synchronize()
    for o, s in zip(outs, singles):
        assert np.array_equal(o.cpu().numpy(), s)


def test_post_needs_the_five_level_pyramid(converter):
    raw, p = _frame()
    p.levels = 4
    with pytest.raises(g.GlsError) as e:
        converter.demosaic(raw, p, postProcess=True)
    assert e.value.code == g.GLS_ERR_INVALID_ARG


@pytest.mark.skipif(not R.available(), reason="reference kernels not built (make -C oracle ref)")
def test_post_vs_reference_kernels(converter):
    # the same planes through the reference's own post-processing kernels
    raw, p = _frame(256, 256, iso=1600, seed=17)
    out = converter.demosaic(raw, p, postProcess=True)
    den, grad = _planes(converter)
    rgb = converter.demosaic(raw, p).astype(np.float32)
    ref, _ = R.postprocess(den, grad, rgb, p, int(raw[0, 0]))
    q, m = _p999(out, ref)
    assert q <= 5e-6 and m <= 2e-4, (q, m)
    # and end to end: raw -> display sRGB through the reference kernels
    ref_e2e, _ = R.demosaic_post(raw, p)
    orc = O.postprocess(*_oracle_planes(raw, p), p, int(raw[0, 0]))[0]
    ps_cuda = scene.psnr(out[..., :3], ref_e2e[..., :3])
    ps_orc = scene.psnr(orc[..., :3], ref_e2e[..., :3])
    assert ps_cuda >= 55.0 and ps_cuda >= ps_orc - 3.0, (ps_cuda, ps_orc)


def _oracle_planes(raw, p):
    st = O.raw_pipeline(raw, p, denoise=True, f64=False, stages=True)
    den = O.pyramid_denoise(st["despeckled"], st["gradient"], p, f64=False, levels_out=True)["levels"]
    return den, st["gradient"], st["out"]
