"""ctypes binding of oracle/_ref/libglsref.so: the reference's own Metal
kernels (demosaic.metal) compiled as C++ and run on the CPU, stage by stage
(see oracle/ref_harness.cpp). Built by `make -C oracle ref` where the
reference tree is present; the shared object travels with the repository
snapshot, so tests that need it skip only where it was never built."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from glasscamerapublic_b200 import DemosaicParams

REF_LIB = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libglsref.so"
_lib = None


def available() -> bool:
    return REF_LIB.exists()


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        L = C.CDLL(str(REF_LIB))
        fp = C.POINTER(C.c_float)
        dp = C.POINTER(C.c_double)
        P = C.POINTER(DemosaicParams)
        L.ref_scale.argtypes = [C.c_void_p, C.c_int, C.c_int, P, fp]
        L.ref_sobel_blur.argtypes = [fp, C.c_int, C.c_int, P, fp]
        L.ref_raw_denoise.argtypes = [fp, fp, C.c_int, C.c_int, P, fp]
        L.ref_demosaic_rgb.argtypes = [fp, fp, C.c_int, C.c_int, P, fp]
        L.ref_transform.argtypes = [fp, C.c_int, C.c_int, fp, fp]
        L.ref_despeckle.argtypes = [fp, C.c_int, C.c_int, P, fp]
        L.ref_pyramid_denoise.argtypes = [fp, fp, C.c_int, C.c_int, P, fp, fp, dp]
        L.ref_raw_pipeline.argtypes = [C.c_void_p, C.c_int, C.c_int, P, C.c_int, fp]
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_calibration_fill.argtypes = [C.c_int, P]
        L.ref_calibration_fill.restype = C.c_int
        L.ref_noise_tables.argtypes = [C.c_uint, C.POINTER(C.c_int32), fp]
        L.ref_postprocess.argtypes = [fp, fp, fp, C.c_int, C.c_int, P, C.c_uint, fp, fp]
        L.ref_demosaic_post.argtypes = [C.c_void_p, C.c_int, C.c_int, P, C.c_int, fp, fp]
        L.ref_raw_noise_stats.argtypes = [fp, C.c_int, C.c_int, C.c_int, fp, fp]
        L.ref_ycc_noise_stats.argtypes = [fp, C.c_int, C.c_int, fp]
        L.ref_measure_raw_nlf.argtypes = [fp, fp, C.c_int, C.c_int, C.c_float, fp, fp]
        L.ref_measure_ycc_nlf.argtypes = [fp, C.c_int, C.c_int, C.c_float, fp, fp]
        _lib = L
    return _lib


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def scale(raw, p):
    raw = np.ascontiguousarray(raw, np.uint16)
    h, w = raw.shape
    out = np.zeros((h, w), np.float32)
    lib().ref_scale(raw.ctypes.data, w, h, C.byref(p), _fp(out))
    return out


def sobel_blur(scaled, p):
    s = _f32(scaled)
    h, w = s.shape
    out = np.zeros((h, w, 2), np.float32)
    lib().ref_sobel_blur(_fp(s), w, h, C.byref(p), _fp(out))
    return out


def raw_denoise(scaled, grad, p):
    s, g = _f32(scaled), _f32(grad)
    h, w = s.shape
    out = np.zeros((h, w), np.float32)
    lib().ref_raw_denoise(_fp(s), _fp(g), w, h, C.byref(p), _fp(out))
    return out


def demosaic_rgb(scaled, grad, p):
    s, g = _f32(scaled), _f32(grad)
    h, w = s.shape
    out = np.zeros((h, w, 4), np.float32)
    lib().ref_demosaic_rgb(_fp(s), _fp(g), w, h, C.byref(p), _fp(out))
    return out


def transform(img, m9):
    a = _f32(img)
    m = _f32(np.asarray(m9).ravel())
    h, w = a.shape[:2]
    out = np.zeros((h, w, 4), np.float32)
    lib().ref_transform(_fp(a), w, h, _fp(m), _fp(out))
    return out


def despeckle(ycc, p):
    a = _f32(ycc)
    h, w = a.shape[:2]
    out = np.zeros((h, w, 4), np.float32)
    lib().ref_despeckle(_fp(a), w, h, C.byref(p), _fp(out))
    return out


def pyramid_denoise(ycc, grad, p):
    a, g = _f32(ycc), _f32(grad)
    h, w = a.shape[:2]
    out = np.zeros((h, w, 4), np.float32)
    bases = np.zeros((p.levels, 25, 8), np.float64)
    lib().ref_pyramid_denoise(_fp(a), _fp(g), w, h, C.byref(p), _fp(out), None,
                              bases.ctypes.data_as(C.POINTER(C.c_double)))
    return out, bases


def raw_pipeline(raw, p, denoise=True):
    raw = np.ascontiguousarray(raw, np.uint16)
    h, w = raw.shape
    out = np.zeros((h, w, 4), np.float32)
    assert lib().ref_raw_pipeline(raw.ctypes.data, w, h, C.byref(p), int(denoise), _fp(out)) == 0
    return out


def noise_tables(seed):
    """Noise2D::randomSeed + initGradients (SimplexNoise.hpp) of the reference."""
    perm = np.zeros(514, np.int32)
    grad = np.zeros((514, 2), np.float32)
    lib().ref_noise_tables(seed, perm.ctypes.data_as(C.POINTER(C.c_int32)), _fp(grad))
    return perm, grad


def postprocess(den_levels, grad, rgb, p, seed):
    """The reference's post-processing kernels (demosaic.metal:1292-1723) in
    the host order of raw_converter.cpp; arguments as _oracle.postprocess."""
    rgb, grad = _f32(rgb), _f32(grad)
    h, w = rgb.shape[:2]
    den = None
    if den_levels is not None:
        den = np.concatenate([_f32(d).ravel() for d in den_levels])
    out = np.zeros((h, w, 4), np.float32)
    st = np.zeros(6, np.float32)
    rc = lib().ref_postprocess(None if den is None else _fp(den), _fp(grad), _fp(rgb), w, h, C.byref(p), seed,
                               _fp(out), _fp(st))
    assert rc == 0, rc
    return out, st


def demosaic_post(raw, p, denoise=True):
    """RawConverter::demosaic(raw, p, noiseReduction, postProcess=true) end
    to end through the reference kernels. Returns (sRGB RGBA, stats)."""
    raw = np.ascontiguousarray(raw, np.uint16)
    h, w = raw.shape
    out = np.zeros((h, w, 4), np.float32)
    st = np.zeros(6, np.float32)
    rc = lib().ref_demosaic_post(raw.ctypes.data, w, h, C.byref(p), int(denoise), _fp(out), _fp(st))
    assert rc == 0, rc
    return out, st


def raw_noise_stats(scaled, pattern):
    """basicRawNoiseStatistics: (mean, var), each (h/2, w/2, 4)."""
    s = _f32(scaled)
    h, w = s.shape
    mean = np.zeros((h // 2, w // 2, 4), np.float32)
    var = np.zeros((h // 2, w // 2, 4), np.float32)
    lib().ref_raw_noise_stats(_fp(s), w, h, int(pattern), _fp(mean), _fp(var))
    return mean, var


def ycc_noise_stats(img):
    """basicNoiseStatistics: (h, w, 4) = mean Y, var Y, var Cb, var Cr."""
    a = _f32(img)
    h, w = a.shape[:2]
    st = np.zeros((h, w, 4), np.float32)
    lib().ref_ycc_noise_stats(_fp(a), w, h, _fp(st))
    return st


def measure_raw_nlf(mean, var, raw_w, raw_h, exposure=1.0):
    """RawConverter::MeasureRawNLF over given statistics: (a[4], b[4])."""
    a = np.zeros(4, np.float32)
    b = np.zeros(4, np.float32)
    lib().ref_measure_raw_nlf(_fp(_f32(mean)), _fp(_f32(var)), raw_w, raw_h, exposure, _fp(a), _fp(b))
    return a, b


def measure_ycc_nlf(stats, exposure=1.0):
    """PyramidProcessor::MeasureYCbCrNLF over given statistics: (a[3], b[3])."""
    st = _f32(stats)
    h, w = st.shape[:2]
    a = np.zeros(3, np.float32)
    b = np.zeros(3, np.float32)
    lib().ref_measure_ycc_nlf(_fp(st), w, h, exposure, _fp(a), _fp(b))
    return a, b


class iPhone14WideCalibration:
    """The reference's own iPhone14WideCalibration<5> (nlfFromIso,
    getDenoiseParameters, buildDemosaicParameters; oracle/ref_calib.cpp) as
    a CameraCalibration for scene.make_params: the parameter block comes
    from the reference's code, not from the library under test."""

    def __init__(self, levels: int = 5):
        self.levels = levels

    def getDemosaicParameters(self, iso: int, params: DemosaicParams | None = None) -> DemosaicParams:
        p = params if params is not None else DemosaicParams()
        rc = lib().ref_calibration_fill(int(iso), C.byref(p))
        if rc != 0:
            raise ValueError(f"reference calibration rejected ISO {iso} (code {rc})")
        p.levels = self.levels
        return p
