"""DNG ingest through the C ABI: gls::image::read_dng_file
(pipelineTest.cpp:114-115) and CameraCalibration::getDemosaicParameters
(CameraCalibration.cpp:25-58) for Python callers."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import CAMERA_IPHONE14_WIDE, DemosaicParams, DngInfo, check, lib

COMPRESSION_NONE = 1
COMPRESSION_LJ92 = 7


def read_dng(path: str):
    """(raw uint16 (h, w), DngInfo)."""
    info = DngInfo()
    p = str(path).encode()
    check(lib().gls_dng_read(p, C.byref(info), None, 0))
    raw = np.empty((info.height, info.width), np.uint16)
    check(lib().gls_dng_read(p, C.byref(info), C.c_void_p(raw.ctypes.data), info.width))
    return raw, info


def write_dng(path: str, raw: np.ndarray, info: DngInfo, compression: int = COMPRESSION_LJ92, tile: int = 256):
    raw = np.ascontiguousarray(raw, np.uint16)
    info.height, info.width = raw.shape
    check(lib().gls_dng_write(str(path).encode(), C.byref(info), C.c_void_p(raw.ctypes.data), raw.shape[1],
                              int(compression), int(tile)))


def camera(info: DngInfo) -> int:
    return int(lib().gls_dng_camera(C.byref(info)))


def demosaic_params(info: DngInfo, xyz_rgb=None, camera_id: int | None = None) -> DemosaicParams:
    """getDemosaicParameters: the DNG's levels, pattern, colour and white
    balance, and the camera's noise model at the DNG's ISO."""
    p = DemosaicParams()
    cid = camera(info) if camera_id is None else camera_id
    if cid < 0:
        cid = CAMERA_IPHONE14_WIDE
    xr = None
    if xyz_rgb is not None:
        xr = (C.c_float * 9)(*np.asarray(xyz_rgb, np.float32).ravel())
    check(lib().gls_dng_demosaic_params(C.byref(info), xr, int(cid), C.byref(p)))
    return p
