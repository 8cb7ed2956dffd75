"""GlassCamera raw-image path on B200 (sm_100a).

Python mirror of the C ABI in include/glscam.h, loaded through ctypes from
the in-tree ``libglscam.so``. The native library is the product; this
module only binds it. There is no CPU fallback: if the library or a CUDA
device is missing, calls fail with :class:`GlsError`.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libglscam.so"

GLS_OK = 0
GLS_ERR_INVALID_ARG = 1
GLS_ERR_OOM = 2
GLS_ERR_CUDA = 3
GLS_ERR_TIMEOUT = 4
GLS_ERR_DEGENERATE = 5
GLS_ERR_UNSUPPORTED = 6
GLS_ERR_RANGE = 7

GRBG, GBRG, RGGB, BGGR = 0, 1, 2, 3
MAX_LEVELS = 5
F32, F16, U16 = 0, 1, 2

DENOISE = 1 << 0
POSTPROCESS = 1 << 1
FP16_STORAGE = 1 << 2
HOST_IO = 1 << 3
SYNC = 1 << 4
GRAPH = 1 << 6
SURF_CORRECTED = 1 << 7
PERSISTENT = 1 << 8
BM_TENSOR = 1 << 9
HOST_PCA = 1 << 5

PLANE_SCALED_RAW = 0
PLANE_GRADIENT = 1
PLANE_DEMOSAIC = 2
PLANE_DESPECKLED = 3
PLANE_OUTPUT = 4
PLANE_ADJ_DESPECKLED = 5
PLANE_NLF_MEAN = 6
PLANE_NLF_VAR = 7
PLANE_DENOISED_L0 = 8
PLANE_NLF_STATS = 13
SURF_PLANE_INTEGRAL = 0
ADJ_NPARAMS = 32
ADJ_LUMA, ADJ_CHROMA, ADJ_NLF_AY, ADJ_NLF_BY, ADJ_NLF_AC, ADJ_NLF_BC = 0, 5, 10, 15, 20, 25
ADJ_RAW_GREEN_A, ADJ_RAW_GREEN_B = 30, 31

CAMERA_IPHONE14_WIDE = 0


class DenoiseParams(C.Structure):
    _fields_ = [(n, C.c_float) for n in
                ("luma", "chroma", "chroma_boost", "gradient_boost", "gradient_threshold", "sharpening")]


class YCbCrNLF(C.Structure):
    _fields_ = [("a", C.c_float * 3), ("b", C.c_float * 3)]


class RawNLF(C.Structure):
    _fields_ = [("a", C.c_float * 4), ("b", C.c_float * 4)]


class RgbConversionParams(C.Structure):
    _fields_ = [
        ("contrast", C.c_float),
        ("saturation", C.c_float),
        ("tone_curve_slope", C.c_float),
        ("exposure_bias", C.c_float),
        ("blacks", C.c_float),
        ("local_tone_mapping", C.c_int32),
    ]


class LtmParams(C.Structure):
    _fields_ = [
        ("eps", C.c_float),
        ("shadows", C.c_float),
        ("highlights", C.c_float),
        ("detail", C.c_float * 3),
    ]


class DemosaicParams(C.Structure):
    _fields_ = [
        ("bayer_pattern", C.c_int32),
        ("black_level", C.c_float),
        ("white_level", C.c_float),
        ("exposure_multiplier", C.c_float),
        ("lens_shading_correction", C.c_float),
        ("scale_mul", C.c_float * 4),
        ("rgb_cam", C.c_float * 9),
        ("xyz_rgb", C.c_float * 9),
        ("high_noise_image", C.c_int32),
        ("raw_denoise_strength", C.c_float),
        ("raw_nlf", RawNLF),
        ("pyramid_nlf", YCbCrNLF * MAX_LEVELS),
        ("denoise", DenoiseParams * MAX_LEVELS),
        ("levels", C.c_int32),
        ("iso", C.c_int32),
        ("rgb_conversion", RgbConversionParams),
        ("ltm", LtmParams),
    ]


class DngInfo(C.Structure):
    """gls_dng_info: a DNG's raw layout and the metadata the parameters
    are built from."""
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("bits_per_sample", C.c_int32),
                ("compression", C.c_int32), ("cfa_pattern", C.c_uint8 * 4), ("bayer_pattern", C.c_int32),
                ("black_level", C.c_float), ("white_level", C.c_float), ("baseline_exposure", C.c_float),
                ("has_color_matrix1", C.c_int32), ("has_color_matrix2", C.c_int32),
                ("has_as_shot_neutral", C.c_int32), ("color_matrix1", C.c_float * 9),
                ("color_matrix2", C.c_float * 9), ("as_shot_neutral", C.c_float * 3),
                ("calibration_illuminant1", C.c_int32), ("calibration_illuminant2", C.c_int32),
                ("iso", C.c_int32), ("exposure_time", C.c_float), ("active_area", C.c_int32 * 4),
                ("make", C.c_char * 64), ("model", C.c_char * 64), ("lens_model", C.c_char * 96)]


class ImageView(C.Structure):
    _fields_ = [
        ("data", C.c_void_p),
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("channels", C.c_int32),
        ("dtype", C.c_int32),
        ("stride_bytes", C.c_size_t),
    ]


class FrameDesc(C.Structure):
    _fields_ = [
        ("raw", C.c_void_p),
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("raw_stride_bytes", C.c_size_t),
        ("params", C.POINTER(DemosaicParams)),
        ("out", ImageView),
    ]


class KernelStat(C.Structure):
    _fields_ = [("name", C.c_char_p), ("launches", C.c_uint64), ("ms", C.c_double)]


# gls_keypoint / gls_match as numpy record types (the reference's KeyPoint
# and DMatch layouts)
KEYPOINT_DTYPE = np.dtype([("x", np.float32), ("y", np.float32), ("size", np.float32), ("angle", np.float32),
                           ("response", np.float32), ("octave", np.int32), ("class_id", np.int32)])
MATCH_DTYPE = np.dtype([("query_idx", np.int32), ("train_idx", np.int32), ("distance", np.float32)])


class GlsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"gls status {code}: {msg}")
        self.code = code


# every symbol include/glscam.h declares: name -> (restype, argtypes)
_SIGNATURES = {
    "gls_last_error_message": (C.c_char_p, []),
    "gls_version": (C.c_char_p, []),
    "gls_device_memory": (C.c_int, [C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.c_int32]),
    "gls_persistent_selftest": (C.c_int, [C.c_int32, C.c_int64, C.POINTER(C.c_int32)]),
    "gls_converter_create": (C.c_int, [C.c_int32, C.c_void_p, C.c_size_t, C.c_int32, C.POINTER(C.c_void_p)]),
    "gls_converter_destroy": (C.c_int, [C.c_void_p]),
    "gls_demosaic": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_size_t,
                               C.POINTER(DemosaicParams), C.c_uint32, C.POINTER(ImageView), C.c_void_p]),
    "gls_demosaic_batch": (C.c_int, [C.c_void_p, C.POINTER(FrameDesc), C.c_int32, C.c_uint32, C.c_void_p]),
    "gls_pyramid_denoise": (C.c_int, [C.c_void_p, C.POINTER(ImageView), C.POINTER(ImageView),
                                      C.POINTER(DemosaicParams), C.c_uint32, C.POINTER(ImageView), C.c_void_p]),
    "gls_converter_plane": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(ImageView)]),
    "gls_converter_pca_basis": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_float)]),
    "gls_copy_view": (C.c_int, [C.POINTER(ImageView), C.POINTER(ImageView), C.c_int32, C.c_void_p]),
    "gls_pca_basis_noalloc": (C.c_int, [C.POINTER(ImageView), C.c_void_p, C.c_void_p]),
    "gls_converter_set_profiling": (C.c_int, [C.c_void_p, C.c_int32]),
    "gls_converter_stats": (C.c_int, [C.c_void_p, C.POINTER(KernelStat), C.c_int32, C.POINTER(C.c_int32)]),
    "gls_converter_reset_stats": (C.c_int, [C.c_void_p]),
    "gls_block_match_tiles": (C.c_int, [C.POINTER(C.c_int32), C.c_int32, C.POINTER(C.c_int32)]),
    "gls_grain_tables": (C.c_int, [C.c_uint32, C.POINTER(C.c_int32), C.POINTER(C.c_float)]),
    "gls_find_bursts": (C.c_int, [C.POINTER(C.c_char_p), C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "gls_convert_to_grayscale": (C.c_int, [C.POINTER(ImageView), C.POINTER(C.c_float), C.POINTER(ImageView),
                                           C.c_void_p]),
    "gls_write_tiff_rgb8": (C.c_int, [C.c_char_p, C.POINTER(ImageView), C.c_void_p]),
    "gls_dng_read": (C.c_int, [C.c_char_p, C.POINTER(DngInfo), C.c_void_p, C.c_size_t]),
    "gls_dng_write": (C.c_int, [C.c_char_p, C.POINTER(DngInfo), C.c_void_p, C.c_size_t, C.c_int32, C.c_int32]),
    "gls_dng_demosaic_params": (C.c_int, [C.POINTER(DngInfo), C.c_void_p, C.c_int32, C.POINTER(DemosaicParams)]),
    "gls_dng_camera": (C.c_int32, [C.POINTER(DngInfo)]),
    "gls_measure_raw_nlf": (C.c_int, [C.c_void_p, C.POINTER(ImageView), C.c_int32, C.c_float, C.POINTER(RawNLF),
                                      C.c_void_p]),
    "gls_measure_ycbcr_nlf": (C.c_int, [C.c_void_p, C.POINTER(ImageView), C.c_float, C.POINTER(YCbCrNLF),
                                        C.c_void_p]),
    "gls_converter_noise_model": (C.c_int, [C.c_void_p, C.POINTER(RawNLF), C.POINTER(YCbCrNLF), C.c_int32,
                                            C.POINTER(C.c_int32)]),
    "gls_calibration_fill": (C.c_int, [C.c_int32, C.c_int32, C.POINTER(DemosaicParams)]),
    "gls_gaussian_bilinear_taps": (C.c_int, [C.c_float, C.POINTER(C.c_float), C.c_int32, C.POINTER(C.c_int32)]),
    "gls_demosaic_denoise_vjp": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_size_t,
                                           C.POINTER(DemosaicParams), C.POINTER(ImageView), C.c_uint32,
                                           C.POINTER(C.c_double), C.POINTER(C.c_float), C.c_void_p]),
    "gls_pyramid_denoise_vjp": (C.c_int, [C.c_void_p, C.POINTER(ImageView), C.POINTER(ImageView),
                                          C.POINTER(DemosaicParams), C.POINTER(ImageView), C.c_uint32,
                                          C.POINTER(C.c_float), C.POINTER(ImageView), C.c_void_p]),
    "gls_surf_create": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_float,
                                  C.POINTER(C.c_void_p)]),
    "gls_surf_destroy": (C.c_int, [C.c_void_p]),
    "gls_surf_detect_and_compute": (C.c_int, [C.c_void_p, C.POINTER(ImageView), C.c_int32, C.c_uint32, C.c_void_p]),
    "gls_surf_features": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                                    C.POINTER(C.c_int32), C.c_void_p]),
    "gls_surf_load_features": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_uint32,
                                         C.c_void_p]),
    "gls_surf_plane":(C.c_int, [C.c_void_p, C.c_int32, C.POINTER(ImageView)]),
    "gls_surf_match": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_int32, C.POINTER(C.c_int32),
                                 C.c_void_p]),
    "gls_surf_find_homography": (C.c_int, [C.c_void_p, C.c_float, C.c_int32, C.POINTER(C.c_float),
                                           C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_void_p]),
    "gls_find_homography": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_int32, C.c_float, C.c_int32,
                                      C.POINTER(C.c_float), C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_void_p]),
    "gls_surf_register_frames": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.c_int32, C.POINTER(C.c_int32),
                                           C.c_int32, C.c_float, C.c_int32, C.c_int32, C.POINTER(C.c_float),
                                           C.c_void_p]),
    "gls_scale_homography": (C.c_int, [C.POINTER(C.c_float), C.c_float, C.POINTER(C.c_float)]),
    "gls_raw_channels": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_size_t, C.c_int32, C.c_float,
                                   C.c_float, C.c_float, C.c_uint32, C.POINTER(ImageView), C.c_uint32, C.c_void_p]),
    "gls_register_and_fuse": (C.c_int, [C.POINTER(ImageView), C.POINTER(ImageView), C.POINTER(ImageView),
                                        C.POINTER(C.c_float), C.c_int32, C.c_void_p]),
    "gls_fuse_pyramid": (C.c_int, [C.c_void_p, C.POINTER(ImageView), C.c_int32, C.POINTER(C.c_float), C.c_int32,
                                   C.c_float, C.POINTER(ImageView), C.c_void_p]),
    "gls_register_image": (C.c_int, [C.POINTER(ImageView), C.POINTER(ImageView), C.POINTER(C.c_float), C.c_void_p]),
}

_lib = None


def lib() -> C.CDLL:
    """The loaded native library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise GlsError(GLS_ERR_UNSUPPORTED,
                           f"{LIB_PATH} is missing: build it with `python -m glasscamerapublic_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code: int) -> None:
    if code != GLS_OK:
        msg = lib().gls_last_error_message().decode(errors="replace")
        raise GlsError(code, msg)


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)


def device_memory(reset_peak: bool = False) -> tuple[int, int]:
    """(current, peak) bytes of device memory the library holds (all devices)."""
    cur, peak = C.c_uint64(0), C.c_uint64(0)
    check(lib().gls_device_memory(C.byref(cur), C.byref(peak), 1 if reset_peak else 0))
    return int(cur.value), int(peak.value)


def block_match_tiles() -> list:
    """The FP16 block matcher's autotuned tile variants: [(w, h, variant)],
    variant = 10 x thread rows + pixels per thread (84, 162: 32x32-pixel
    tiles; 44, 82: 32x16)."""
    buf = (C.c_int32 * 192)()
    n = C.c_int32(0)
    check(lib().gls_block_match_tiles(buf, 64, C.byref(n)))
    return [(buf[3 * i], buf[3 * i + 1], buf[3 * i + 2]) for i in range(min(n.value, 64))]


from .api import CameraCalibration, iPhone14WideCalibration, RawConverter, PyramidProcessor  # noqa: E402

__all__ = [
    "lib", "check", "GlsError", "DemosaicParams", "ImageView", "FrameDesc", "DenoiseParams",
    "RawConverter", "PyramidProcessor", "CameraCalibration", "iPhone14WideCalibration",
]
