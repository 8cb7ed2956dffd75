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


def read_dng_into(path: str, raw_ptr: int, stride_elems: int) -> DngInfo:
    """gls_dng_read into caller memory (e.g. a pinned buffer) of at least
    height x stride_elems uint16."""
    info = DngInfo()
    check(lib().gls_dng_read(str(path).encode(), C.byref(info), C.c_void_p(raw_ptr), int(stride_elems)))
    return info


def convert_files(converter, paths, postProcess: bool = True, stream=None):
    """pipelineTest's demosaicFile over many files (pipelineTest.cpp:110-175),
    pipelined: a host thread reads and decodes the next DNG into a pinned
    buffer while the GPU converts the current one (demosaic, noise
    reduction and, with postProcess, display post-processing; FP16 storage)
    with its copies on the converter's copy streams. Yields (path, RGBA
    FP16 pinned host tensor); each yielded tensor is reused two files
    later. The files must share one size."""
    from concurrent.futures import ThreadPoolExecutor

    import torch

    paths = [str(p) for p in paths]
    if not paths:
        return
    info0 = DngInfo()
    check(lib().gls_dng_read(paths[0].encode(), C.byref(info0), None, 0))
    h, w = info0.height, info0.width
    raws = [torch.empty((h, w), dtype=torch.int16).pin_memory() for _ in range(2)]
    outs = [torch.empty((h, w, 4), dtype=torch.float16).pin_memory() for _ in range(2)]
    s = stream if stream is not None else torch.cuda.Stream()
    with ThreadPoolExecutor(max_workers=1) as ex:
        nxt = ex.submit(read_dng_into, paths[0], raws[0].data_ptr(), w)
        for i, path in enumerate(paths):
            info = nxt.result()
            if (info.height, info.width) != (h, w):
                raise ValueError(f"{path}: {info.width}x{info.height}, expected {w}x{h}")
            if i + 1 < len(paths):
                nxt = ex.submit(read_dng_into, paths[i + 1], raws[(i + 1) % 2].data_ptr(), w)
            p = demosaic_params(info)
            converter.demosaic_batch([raws[i % 2]], [p], [outs[i % 2]], fp16=True, out_fp16=True, stream=s,
                                     postProcess=postProcess)
            yield path, outs[i % 2]
