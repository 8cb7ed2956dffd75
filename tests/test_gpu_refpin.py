"""GPU path against the reference's own kernels (oracle/_ref/libglsref.so:
MetalPipeline/demosaic.metal compiled for the CPU), end to end through the
C ABI.

The reference computes most stages in half precision (texture2d<half>
kernels); the CUDA FP32 path computes them in FP32, the FP16-storage path
stores planes in half and computes in FP32. Both are compared to the
reference kernels' raw -> linear RGB output by PSNR over RGB in [0, ~1.1]:
  * FP32 path: >= 55 dB, and within 3 dB of the CPU oracle's FP32 run's
    PSNR against the same reference output;
  * FP16-storage path: >= 50 dB.
"""
import numpy as np
import pytest

import _oracle as O
import _ref as R
from glasscamerapublic_b200 import scene

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not R.available(), reason="reference kernels not built (make -C oracle ref)")]


@pytest.mark.parametrize("iso,pattern", [(200, 2), (1600, 2), (1600, 0), (400, 3)])
def test_cuda_paths_vs_reference_kernels(converter, iso, pattern):
    wl = scene.Workload("refpin", 320, 240, levels=4, gain=0.8, read=3.0, iso=iso, seed=iso + pattern,
                        pattern=pattern)
    raw, clean = scene.make_raw(wl)
    p = scene.make_params(wl)
    ref = R.raw_pipeline(raw, p, denoise=True)[..., :3]
    orc = O.raw_pipeline(raw, p, denoise=True, f64=False)["out"][..., :3]
    out32 = converter.demosaic(raw, p, noiseReduction=True)[..., :3]
    out16 = converter.demosaic(raw, p, noiseReduction=True, fp16=True)[..., :3]
    ps_orc = scene.psnr(orc, ref)
    ps32 = scene.psnr(out32, ref)
    ps16 = scene.psnr(out16, ref)
    assert ps32 >= 55.0, (ps32, ps_orc)
    assert ps32 >= ps_orc - 3.0, (ps32, ps_orc)
    assert ps16 >= 50.0, ps16


def test_cuda_front_end_vs_reference_kernels(converter):
    # no denoise: scale, gradients, demosaic, highlights, despeckle, transforms
    wl = scene.Workload("refpin", 256, 192, levels=4, gain=0.8, read=3.0, iso=200, seed=5)
    raw, clean = scene.make_raw(wl)
    p = scene.make_params(wl)
    ref = R.raw_pipeline(raw, p, denoise=False)[..., :3]
    out32 = converter.demosaic(raw, p, noiseReduction=False)[..., :3]
    d = np.abs(out32.astype(np.float64) - ref)
    # the reference rounds scaleRawData and the Sobel image to half
    assert float(np.quantile(d, 0.999)) <= 1e-3, float(np.quantile(d, 0.999))
    assert scene.psnr(out32, ref) >= 55.0
