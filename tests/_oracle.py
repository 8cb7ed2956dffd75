"""ctypes binding of the CPU oracle (oracle/liboracle.so) for the tests.

The oracle is the checker: tests compare the CUDA library with it. It is
built from oracle/Makefile on first use when the shared object is missing.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

from glasscamerapublic_b200 import DemosaicParams

ROOT = Path(__file__).resolve().parents[1]
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "liboracle.so"

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not ORACLE_LIB.exists():
            subprocess.run(["make", "-C", str(ORACLE_DIR)], check=True, capture_output=True)
        L = C.CDLL(str(ORACLE_LIB))
        fp = C.POINTER(C.c_float)
        dp = C.POINTER(C.c_double)
        L.orc_raw_pipeline.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_size_t, C.POINTER(DemosaicParams),
                                       C.c_int, C.c_int, fp, fp, fp, fp, fp, dp]
        L.orc_pyramid_denoise.argtypes = [fp, fp, C.c_int, C.c_int, C.POINTER(DemosaicParams), C.c_int, fp, fp, dp]
        L.orc_gaussian_taps.argtypes = [C.c_float, fp, C.c_int, C.POINTER(C.c_int)]
        L.orc_cam_ycbcr.argtypes = [fp, fp, fp, fp]
        L.orc_bayer_roundtrip.argtypes = [fp, C.c_int, C.c_int, C.c_int, fp, fp]
        L.orc_downsample.argtypes = [fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, fp]
        L.orc_pca_basis.argtypes = [fp, C.c_int, C.c_int, dp]
        L.orc_jacobi.argtypes = [C.c_int, dp, dp, dp]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_pyramid_loss.argtypes = [fp, fp, C.c_int, C.c_int, C.POINTER(DemosaicParams), dp, dp, fp, C.c_int, dp]
        L.orc_postprocess.argtypes = [fp, fp, fp, C.c_int, C.c_int, C.POINTER(DemosaicParams), C.c_uint, C.c_int,
                                      fp, fp]
        _lib = L
    return _lib


def _fp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def raw_pipeline(raw: np.ndarray, p: DemosaicParams, denoise: bool = True, f64: bool = True,
                 stages: bool = False, bases: bool = False):
    raw = np.ascontiguousarray(raw, dtype=np.uint16)
    h, w = raw.shape
    out = np.zeros((h, w, 4), np.float32)
    st = {}
    if stages:
        st = {"scaled": np.zeros((h, w), np.float32), "gradient": np.zeros((h, w, 2), np.float32),
              "demosaic": np.zeros((h, w, 4), np.float32), "despeckled": np.zeros((h, w, 4), np.float32)}
    b = np.zeros((p.levels, 25, 8), np.float64) if bases else None
    rc = lib().orc_raw_pipeline(raw.ctypes.data, w, h, w, C.byref(p), int(denoise), int(f64), _fp(out),
                                _fp(st.get("scaled")), _fp(st.get("gradient")), _fp(st.get("demosaic")),
                                _fp(st.get("despeckled")), _dp(b))
    assert rc == 0
    res = {"out": out, **st}
    if bases:
        res["bases"] = b
    return res


def pyramid_denoise(ycc: np.ndarray, grad: np.ndarray, p: DemosaicParams, f64: bool = True, levels_out=False):
    ycc = np.ascontiguousarray(ycc, np.float32)
    grad = np.ascontiguousarray(grad, np.float32)
    h, w = ycc.shape[:2]
    out = np.zeros((h, w, 4), np.float32)
    tot = sum((w >> i) * (h >> i) * 4 for i in range(p.levels))
    lv = np.zeros(tot, np.float32) if levels_out else None
    b = np.zeros((p.levels, 25, 8), np.float64)
    assert lib().orc_pyramid_denoise(_fp(ycc), _fp(grad), w, h, C.byref(p), int(f64), _fp(out), _fp(lv), _dp(b)) == 0
    res = {"out": out, "bases": b}
    if levels_out:
        levels, off = [], 0
        for i in range(p.levels):
            n = (w >> i) * (h >> i) * 4
            levels.append(lv[off:off + n].reshape(h >> i, w >> i, 4))
            off += n
        res["levels"] = levels
    return res


def gaussian_taps(radius: float) -> np.ndarray:
    buf = np.zeros(64 * 3, np.float32)
    n = C.c_int()
    assert lib().orc_gaussian_taps(radius, _fp(buf), 64, C.byref(n)) == 0
    return buf[: 3 * n.value].reshape(-1, 3)


def cam_ycbcr(rgb_cam, xyz_rgb):
    a = np.asarray(rgb_cam, np.float32).ravel().copy()
    b = np.asarray(xyz_rgb, np.float32).ravel().copy()
    f = np.zeros(9, np.float32)
    i = np.zeros(9, np.float32)
    lib().orc_cam_ycbcr(_fp(a), _fp(b), _fp(f), _fp(i))
    return f.reshape(3, 3), i.reshape(3, 3)


def bayer_roundtrip(raw: np.ndarray, pattern: int):
    raw = np.ascontiguousarray(raw, np.float32)
    h, w = raw.shape
    q = np.zeros((h // 2, w // 2, 4), np.float32)
    back = np.zeros((h, w), np.float32)
    lib().orc_bayer_roundtrip(_fp(raw), w, h, pattern, _fp(q), _fp(back))
    return q, back


def downsample(img: np.ndarray, ow: int, oh: int, f64: bool = True):
    img = np.ascontiguousarray(img, np.float32)
    h, w, ch = img.shape
    out = np.zeros((oh, ow, ch), np.float32)
    assert lib().orc_downsample(_fp(img), w, h, ch, ow, oh, int(f64), _fp(out)) == 0
    return out


def pca_basis(img4: np.ndarray) -> np.ndarray:
    img4 = np.ascontiguousarray(img4, np.float32)
    h, w = img4.shape[:2]
    b = np.zeros((25, 8), np.float64)
    lib().orc_pca_basis(_fp(img4), w, h, _dp(b))
    return b


def jacobi(a: np.ndarray):
    a = np.ascontiguousarray(a, np.float64)
    n = a.shape[0]
    ev = np.zeros(n)
    vec = np.zeros((n, n))
    lib().orc_jacobi(n, _dp(a), _dp(ev), _dp(vec))
    return ev, vec


# ---- stage entry points (same inputs as the reference harness's stages)
def _stage_setup(L):
    fp = C.POINTER(C.c_float)
    P = C.POINTER(DemosaicParams)
    L.orc_scale.argtypes = [C.c_void_p, C.c_int, C.c_int, P, C.c_int, fp]
    L.orc_sobel_blur.argtypes = [fp, C.c_int, C.c_int, P, C.c_int, fp]
    L.orc_raw_denoise.argtypes = [fp, fp, C.c_int, C.c_int, P, C.c_int, fp]
    L.orc_demosaic_rgb.argtypes = [fp, fp, C.c_int, C.c_int, P, C.c_int, fp]
    L.orc_despeckle.argtypes = [fp, C.c_int, C.c_int, P, C.c_int, fp]


def stage(name, *arrays, p, w, h, out_shape, f64=False, raw=None):
    L = lib()
    if not hasattr(L, "_stages_ready"):
        _stage_setup(L)
        L._stages_ready = True
    out = np.zeros(out_shape, np.float32)
    args = [(_fp(np.ascontiguousarray(a, np.float32))) for a in arrays]
    keep = [np.ascontiguousarray(a, np.float32) for a in arrays]
    args = [_fp(k) for k in keep]
    fn = getattr(L, "orc_" + name)
    if raw is not None:
        raw = np.ascontiguousarray(raw, np.uint16)
        assert fn(raw.ctypes.data, w, h, C.byref(p), int(f64), _fp(out)) == 0
    else:
        assert fn(*args, w, h, C.byref(p), int(f64), _fp(out)) == 0
    return out


def pyramid_loss(ycc, grad, p: DemosaicParams, bases, y2c, target) -> float:
    """MSE of the FP64 pyramid (bases held fixed) + output transform vs target."""
    ycc = np.ascontiguousarray(ycc, np.float32)
    grad = np.ascontiguousarray(grad, np.float32)
    t = np.ascontiguousarray(target, np.float32)
    b = np.ascontiguousarray(bases, np.float64)
    m = np.ascontiguousarray(np.asarray(y2c, np.float64).ravel())
    h, w = ycc.shape[:2]
    out = C.c_double(0)
    assert lib().orc_pyramid_loss(_fp(ycc), _fp(grad), w, h, C.byref(p), _dp(b), _dp(m), _fp(t), t.shape[2],
                                  C.byref(out)) == 0
    return out.value


def postprocess(den_levels, grad, rgb, p: DemosaicParams, seed: int, f64: bool = False):
    """The display post-processing of one frame (oracle/gls_oracle_post.hpp).
    den_levels: list of 5 (h >> l, w >> l, 4) YCbCr levels, or None without
    noise reduction; grad (h, w, 2); rgb (h, w, 4) linear camera RGB.
    Returns (out (h, w, 4), stats [black, white, shadows, highlights, mean,
    median])."""
    rgb = np.ascontiguousarray(rgb, np.float32)
    grad = np.ascontiguousarray(grad, np.float32)
    h, w = rgb.shape[:2]
    den = None
    if den_levels is not None:
        den = np.concatenate([np.ascontiguousarray(d, np.float32).ravel() for d in den_levels])
    out = np.zeros((h, w, 4), np.float32)
    st = np.zeros(6, np.float32)
    assert lib().orc_postprocess(_fp(den), _fp(grad), _fp(rgb), w, h, C.byref(p), seed, int(f64), _fp(out),
                                 _fp(st)) == 0
    return out, st


def _nlf_setup(L):
    fp = C.POINTER(C.c_float)
    L.orc_raw_noise_stats.argtypes = [fp, C.c_int, C.c_int, C.c_int, fp, fp]
    L.orc_ycc_noise_stats.argtypes = [fp, C.c_int, C.c_int, fp]
    L.orc_measure_raw_nlf.argtypes = [fp, fp, C.c_int, C.c_int, C.c_float, fp, fp]
    L.orc_measure_ycc_nlf.argtypes = [fp, C.c_int, C.c_int, C.c_float, fp, fp]
    L.orc_raw_pipeline_calibrated.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_size_t, C.POINTER(DemosaicParams),
                                              C.c_int, fp, fp, fp]
    L._nlf_ready = True


def _nlf_lib():
    L = lib()
    if not hasattr(L, "_nlf_ready"):
        _nlf_setup(L)
    return L


def raw_noise_stats(scaled, pattern):
    """basicRawNoiseStatistics (FP32): (mean, var), each (h/2, w/2, 4)."""
    s = np.ascontiguousarray(scaled, np.float32)
    h, w = s.shape
    mean = np.zeros((h // 2, w // 2, 4), np.float32)
    var = np.zeros((h // 2, w // 2, 4), np.float32)
    assert _nlf_lib().orc_raw_noise_stats(_fp(s), w, h, int(pattern), _fp(mean), _fp(var)) == 0
    return mean, var


def ycc_noise_stats(img):
    """basicNoiseStatistics (FP32): (h, w, 4) = mean Y, var Y, var Cb, var Cr."""
    a = np.ascontiguousarray(img, np.float32)
    h, w = a.shape[:2]
    st = np.zeros((h, w, 4), np.float32)
    assert _nlf_lib().orc_ycc_noise_stats(_fp(a), w, h, _fp(st)) == 0
    return st


def measure_raw_nlf(mean, var, raw_w, raw_h, exposure=1.0):
    a = np.zeros(4, np.float32)
    b = np.zeros(4, np.float32)
    assert _nlf_lib().orc_measure_raw_nlf(_fp(np.ascontiguousarray(mean, np.float32)),
                                          _fp(np.ascontiguousarray(var, np.float32)), raw_w, raw_h, exposure,
                                          _fp(a), _fp(b)) == 0
    return a, b


def measure_ycc_nlf(stats, exposure=1.0):
    st = np.ascontiguousarray(stats, np.float32)
    h, w = st.shape[:2]
    a = np.zeros(3, np.float32)
    b = np.zeros(3, np.float32)
    assert _nlf_lib().orc_measure_ycc_nlf(_fp(st), w, h, exposure, _fp(a), _fp(b)) == 0
    return a, b


def raw_pipeline_calibrated(raw, p, f64=False):
    """RawConverter::demosaic with calibrateFromImage: (out RGBA, raw NLF
    (a[4], b[4]), pyramid NLF (levels, 2, 3))."""
    raw = np.ascontiguousarray(raw, dtype=np.uint16)
    h, w = raw.shape
    out = np.zeros((h, w, 4), np.float32)
    rn = np.zeros(8, np.float32)
    pn = np.zeros((p.levels, 6), np.float32)
    assert _nlf_lib().orc_raw_pipeline_calibrated(raw.ctypes.data, w, h, w, C.byref(p), int(f64), _fp(out), _fp(rn),
                                                  _fp(pn)) == 0
    return out, (rn[:4], rn[4:]), pn.reshape(p.levels, 2, 3)
