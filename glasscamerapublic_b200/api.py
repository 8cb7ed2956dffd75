"""Python mirror of the reference's RawConverter / PyramidProcessor /
CameraCalibration interface (MetalPipeline/raw_converter.hpp:80-188,
MetalPipeline/pyramid_processor.hpp:23-76, MetalPipeline/CameraCalibration.hpp:24-39),
bound to the C ABI of libglscam.so. Method names follow the reference.

Host inputs are numpy arrays; device inputs are torch CUDA tensors (torch is
only the allocator and stream provider here). All compute runs in the
native library; nothing here computes pixels.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import (BM_TENSOR, DENOISE, F16, F32, FP16_STORAGE, GRAPH, HOST_IO, HOST_PCA, PERSISTENT, POSTPROCESS,
               SYNC,
               CAMERA_IPHONE14_WIDE,
               DemosaicParams, ImageView, FrameDesc, RawNLF, YCbCrNLF, check, lib)


def _stream_handle(stream) -> C.c_void_p:
    if stream is None:
        return C.c_void_p(None)
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(stream.cuda_stream)


class CameraCalibration:
    """CameraCalibration<levels> (CameraCalibration.hpp:24-39) of a built-in camera."""

    camera_id = -1

    def __init__(self, levels: int = 5):
        self.levels = levels

    def getDemosaicParameters(self, iso: int, params: DemosaicParams | None = None) -> DemosaicParams:
        """nlfFromIso(iso) + getDenoiseParameters(iso) into a parameter block."""
        p = params if params is not None else DemosaicParams()
        p.levels = self.levels
        check(lib().gls_calibration_fill(self.camera_id, int(iso), C.byref(p)))
        p.levels = self.levels
        return p

    def nlfFromIso(self, iso: int):
        p = self.getDemosaicParameters(iso)
        return p.raw_nlf, list(p.pyramid_nlf)

    def getDenoiseParameters(self, iso: int):
        p = self.getDemosaicParameters(iso)
        return (bool(p.high_noise_image), p.raw_denoise_strength), list(p.denoise)


class iPhone14WideCalibration(CameraCalibration):
    """iPhone14WideCalibration (MetalPipeline/iPhone14WideCalibration.cpp)."""

    camera_id = CAMERA_IPHONE14_WIDE


def _view_for_array(a, dtype_code: int, channels: int) -> ImageView:
    h, w = a.shape[0], a.shape[1]
    return ImageView(C.c_void_p(_ptr(a)), w, h, channels, dtype_code, _row_stride(a))


def _ptr(a) -> int:
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()


def _row_stride(a) -> int:
    if isinstance(a, np.ndarray):
        return a.strides[0]
    return a.stride(0) * a.element_size()


def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


class RawConverter:
    """RawConverter (raw_converter.hpp:80-188) on a CUDA device."""

    def __init__(self, device: int = 0, calibrateFromImage: bool = False):
        h = C.c_void_p()
        check(lib().gls_converter_create(int(device), None, 0, 1 if calibrateFromImage else 0, C.byref(h)))
        self._h = h
        self.device = device
        self.calibrateFromImage = calibrateFromImage

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().gls_converter_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def demosaic(self, raw, params: DemosaicParams, noiseReduction: bool = True, fp16: bool = False,
                 out=None, out_fp16: bool = False, stream=None, host_pca: bool = False, sync: bool = True,
                 postProcess: bool = False):
        """RawConverter::demosaic(raw, params, noiseReduction, postProcess).

        ``raw``: numpy uint16 (H, W) host array, or a torch CUDA int16/uint16
        tensor. Returns RGBA (H, W, 4): linear camera RGB, or display sRGB in
        [0, 1] with ``postProcess`` (raw_converter.cpp:226-242); a numpy array
        for host input, or ``out`` (a torch CUDA tensor) for device input.
        """
        flags = (DENOISE if noiseReduction else 0) | (FP16_STORAGE if fp16 else 0) | (HOST_PCA if host_pca else 0)
        flags |= POSTPROCESS if postProcess else 0
        flags |= SYNC if sync else 0
        dt = F16 if out_fp16 else F32
        h, w = raw.shape[0], raw.shape[1]
        if not _is_torch(raw):
            raw = np.ascontiguousarray(raw, dtype=np.uint16)
            flags |= HOST_IO
            if out is None:
                out = np.empty((h, w, 4), dtype=np.float16 if out_fp16 else np.float32)
        elif out is None:
            import torch
            out = torch.empty((h, w, 4), dtype=torch.float16 if out_fp16 else torch.float32, device=raw.device)
        ov = ImageView(C.c_void_p(_ptr(out)), w, h, 4, dt, _row_stride(out))
        check(lib().gls_demosaic(self._h, C.c_void_p(_ptr(raw)), w, h, _row_stride(raw), C.byref(params), flags,
                                 C.byref(ov), _stream_handle(stream)))
        return out

    def demosaic_batch(self, raws, params_list, outs, fp16: bool = True, noiseReduction: bool = True,
                       out_fp16: bool = True, stream=None, sync: bool = False, host_pca: bool = False,
                       graph: bool = False, postProcess: bool = False, persistent: bool = False,
                       tensor_bm: bool = False):
        """Batched RawConverter::demosaic over frames of uneven sizes.

        ``raws``/``outs``: torch CUDA tensors (device I/O), or host buffers
        (numpy arrays or pinned torch CPU tensors; copied inside the call).
        ``tensor_bm``: the tensor-core block matcher (GLS_BM_TENSOR; stream-
        launched batches, the persistent batch runs the default matcher).
        """
        n = len(raws)
        frames = (FrameDesc * n)()
        host = False
        for i, (r, p, o) in enumerate(zip(raws, params_list, outs)):
            h, w = r.shape[0], r.shape[1]
            host = host or not (_is_torch(r) and r.is_cuda)
            frames[i].raw = C.c_void_p(_ptr(r))
            frames[i].width = w
            frames[i].height = h
            frames[i].raw_stride_bytes = _row_stride(r)
            frames[i].params = C.pointer(p)
            frames[i].out = ImageView(C.c_void_p(_ptr(o)), w, h, 4, F16 if out_fp16 else F32, _row_stride(o))
        flags = (DENOISE if noiseReduction else 0) | (FP16_STORAGE if fp16 else 0) | (SYNC if sync else 0)
        flags |= (HOST_IO if host else 0) | (HOST_PCA if host_pca else 0) | (GRAPH if graph else 0)
        flags |= (POSTPROCESS if postProcess else 0) | (PERSISTENT if persistent else 0)
        flags |= BM_TENSOR if tensor_bm else 0
        check(lib().gls_demosaic_batch(self._h, frames, n, flags, _stream_handle(stream)))
        return outs

    def plane(self, which: int) -> np.ndarray:
        """Host copy of an internal plane of the last call."""
        v = ImageView()
        check(lib().gls_converter_plane(self._h, int(which), C.byref(v)))
        dt = np.float16 if v.dtype == F16 else np.float32
        arr = np.empty((v.height, v.width, v.channels), dtype=dt)
        dst = ImageView(C.c_void_p(arr.ctypes.data), v.width, v.height, v.channels, v.dtype, arr.strides[0])
        check(lib().gls_copy_view(C.byref(v), C.byref(dst), 0, None))
        return arr

    def MeasureRawNLF(self, scaled, bayerPattern: int, exposure_multiplier: float = 1.0, stream=None):
        """RawConverter::MeasureRawNLF (raw_converter.cpp:339-490) on a scaled
        raw frame (a torch CUDA (h, w) float32/float16 tensor): (a[4], b[4])."""
        v = ImageView(C.c_void_p(_ptr(scaled)), scaled.shape[1], scaled.shape[0], 1,
                      F16 if str(scaled.dtype) == "torch.float16" else F32, _row_stride(scaled))
        r = RawNLF()
        check(lib().gls_measure_raw_nlf(self._h, C.byref(v), int(bayerPattern), float(exposure_multiplier),
                                        C.byref(r), _stream_handle(stream)))
        return np.array(r.a[:], np.float32), np.array(r.b[:], np.float32)

    def MeasureYCbCrNLF(self, ycc, exposure_multiplier: float = 1.0, stream=None):
        """PyramidProcessor::MeasureYCbCrNLF (pyramid_processor.cpp:173-324)
        on a YCbCr image (a torch CUDA (h, w, 4) tensor): (a[3], b[3])."""
        v = ImageView(C.c_void_p(_ptr(ycc)), ycc.shape[1], ycc.shape[0], 4,
                      F16 if str(ycc.dtype) == "torch.float16" else F32, _row_stride(ycc))
        r = YCbCrNLF()
        check(lib().gls_measure_ycbcr_nlf(self._h, C.byref(v), float(exposure_multiplier), C.byref(r),
                                          _stream_handle(stream)))
        return np.array(r.a[:], np.float32), np.array(r.b[:], np.float32)

    def noise_model(self):
        """The models the last calibrating call measured: ((a[4], b[4]),
        [(a[3], b[3]) per pyramid level])."""
        r = RawNLF()
        pyr = (YCbCrNLF * 5)()
        n = C.c_int32()
        check(lib().gls_converter_noise_model(self._h, C.byref(r), pyr, 5, C.byref(n)))
        return ((np.array(r.a[:], np.float32), np.array(r.b[:], np.float32)),
                [(np.array(pyr[i].a[:], np.float32), np.array(pyr[i].b[:], np.float32)) for i in range(n.value)])

    def pca_basis(self, level: int) -> np.ndarray:
        b = (C.c_float * 200)()
        check(lib().gls_converter_pca_basis(self._h, int(level), b))
        return np.frombuffer(b, dtype=np.float32).reshape(25, 8).copy()


class PyramidProcessor:
    """PyramidProcessor<levels> (pyramid_processor.hpp:23-76)."""

    def __init__(self, converter: RawConverter | None = None, device: int = 0):
        self.converter = converter if converter is not None else RawConverter(device)

    def denoise(self, ycc, gradient, params: DemosaicParams, fp16: bool = False, host_pca: bool = False):
        """PyramidProcessor::denoise on a YCbCr image (H, W, 4) and its
        gradient (H, W, 2), float32 numpy arrays. Returns denoised YCbCr
        (H, W, 4), w = luma kernel norm."""
        ycc = np.ascontiguousarray(ycc, dtype=np.float32)
        gradient = np.ascontiguousarray(gradient, dtype=np.float32)
        h, w = ycc.shape[:2]
        out = np.empty((h, w, 4), dtype=np.float32)
        yv = _view_for_array(ycc, F32, 4)
        gv = _view_for_array(gradient, F32, 2)
        ov = _view_for_array(out, F32, 4)
        flags = HOST_IO | SYNC | (FP16_STORAGE if fp16 else 0) | (HOST_PCA if host_pca else 0)
        check(lib().gls_pyramid_denoise(self.converter.handle, C.byref(yv), C.byref(gv), C.byref(params), flags,
                                        C.byref(ov), None))
        return out

    def denoise_vjp(self, ycc, gradient, params: DemosaicParams, g_out):
        """Vector-Jacobian product of the FP32 denoise (gls_pyramid_denoise_vjp):
        given g_out = dL/d(denoised Y, Cb, Cr) (H, W, 3|4), returns
        (dL/dtheta [32], dL/d ycc (H, W, 3)), the PCA bases held fixed.
        Float32 numpy arrays."""
        ycc = np.ascontiguousarray(ycc, dtype=np.float32)
        gradient = np.ascontiguousarray(gradient, dtype=np.float32)
        g_out = np.ascontiguousarray(g_out, dtype=np.float32)
        h, w = ycc.shape[:2]
        g_ycc = np.empty((h, w, 3), dtype=np.float32)
        grad = np.zeros(32, np.float32)
        yv = _view_for_array(ycc, F32, 4)
        gv = _view_for_array(gradient, F32, 2)
        ov = _view_for_array(g_out, F32, g_out.shape[2])
        iv = _view_for_array(g_ycc, F32, 3)
        check(lib().gls_pyramid_denoise_vjp(self.converter.handle, C.byref(yv), C.byref(gv), C.byref(params),
                                            C.byref(ov), HOST_IO, grad.ctypes.data_as(C.POINTER(C.c_float)),
                                            C.byref(iv), None))
        return grad, g_ycc
