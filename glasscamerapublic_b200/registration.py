"""Python mirror of the reference's registration and fusion interface
(ImageRegistration/SURF.hpp:45-80, Homography.hpp:26-37,
MetalPipeline/demosaic_kernels.hpp:690-710, PyramidFusion/pyramidFusion.cpp:106-143),
bound to the C ABI of libglscam.so. Method names follow the reference.

Host inputs are numpy arrays; device inputs are torch CUDA tensors (torch is
only the allocator and stream provider). All compute runs in the native
library.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import F16, F32, HOST_IO, KEYPOINT_DTYPE, MATCH_DTYPE, SURF_CORRECTED, SYNC, ImageView, check, lib
from .api import _is_torch, _ptr, _row_stride, _stream_handle

SURF_SLOTS = 32


def _view(a, channels: int) -> ImageView:
    h, w = a.shape[0], a.shape[1]
    if _is_torch(a):
        import torch
        code = F32 if a.dtype == torch.float32 else F16
    else:
        code = F32 if a.dtype == np.float32 else F16
    return ImageView(C.c_void_p(_ptr(a)), w, h, channels, code, _row_stride(a))


class SURF:
    """SURF::makeInstance(ctx, width, height, max_features, nOctaves,
    nOctaveLayers, hessianThreshold) (SURF.hpp:45-47). Results of
    detectAndCompute stay on the GPU in one of SURF_SLOTS feature slots.

    The detector is the reference's, two defects included (the maxima
    interpolation moves x, y and size by the scale offset, SURF.metal:200;
    a set of 33..56 keypoints is only partly described, SURF.cpp:681-693).
    corrected=True solves the interpolation per axis and describes every
    keypoint (GLS_SURF_CORRECTED)."""

    def __init__(self, width: int, height: int, max_features: int = -1, nOctaves: int = 4, nOctaveLayers: int = 2,
                 hessianThreshold: float = 0.02, device: int = 0, corrected: bool = False):
        self._detect_flags = SURF_CORRECTED if corrected else 0
        h = C.c_void_p()
        check(lib().gls_surf_create(device, width, height, max_features, nOctaves, nOctaveLayers,
                                    float(hessianThreshold), C.byref(h)))
        self._h = h
        self.width, self.height = width, height
        self.max_features = max_features
        self._next_slot = 0

    @classmethod
    def makeInstance(cls, width: int, height: int, max_features: int = -1, nOctaves: int = 4,
                     nOctaveLayers: int = 2, hessianThreshold: float = 0.02, device: int = 0) -> "SURF":
        return cls(width, height, max_features, nOctaves, nOctaveLayers, hessianThreshold, device)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().gls_surf_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    @property
    def corrected(self) -> bool:
        """Whether detections use the corrected detector (GLS_SURF_CORRECTED)."""
        return bool(self._detect_flags & SURF_CORRECTED)

    @corrected.setter
    def corrected(self, on: bool):
        self._detect_flags = SURF_CORRECTED if on else 0

    def detect_slot(self, img, slot: int, stream=None, sync: bool = False) -> int:
        """Detection + description of img (F32 H x W, numpy or CUDA tensor)
        into a slot, asynchronously for device input."""
        v = _view(img, 1)
        flags = (HOST_IO if isinstance(img, np.ndarray) else 0) | self._detect_flags
        if sync:
            flags |= SYNC
        check(lib().gls_surf_detect_and_compute(self._h, C.byref(v), slot, flags, _stream_handle(stream)))
        return slot

    def features(self, slot: int, stream=None):
        cap = self.max_features if self.max_features >= 0 else 64000
        kps = np.zeros(cap, KEYPOINT_DTYPE)
        desc = np.zeros((cap, 64), np.float32)
        n = C.c_int32(0)
        check(lib().gls_surf_features(self._h, slot, kps.ctypes.data, desc.ctypes.data, cap, C.byref(n),
                                      _stream_handle(stream)))
        return kps[:n.value].copy(), desc[:n.value].copy()

    def load_features(self, slot: int, kps, desc, stream=None) -> int:
        """Loads keypoints (KEYPOINT_DTYPE records, or their bytes as a
        uint8 CUDA tensor) and descriptors ([n][64] float32, numpy or CUDA)
        into a slot, as features() returned them on another detector."""
        if isinstance(kps, np.ndarray):
            k = np.ascontiguousarray(kps).view(KEYPOINT_DTYPE)
            d = np.ascontiguousarray(desc, np.float32).reshape(-1, 64)
            n, kp, dp, flags = len(k), k.ctypes.data, d.ctypes.data, HOST_IO
        else:
            n = kps.numel() // KEYPOINT_DTYPE.itemsize
            kp, dp, flags = _ptr(kps), _ptr(desc), 0
        if desc.shape[0] != n:
            raise ValueError(f"{n} keypoints but {desc.shape[0]} descriptors")
        check(lib().gls_surf_load_features(self._h, slot, kp, dp, n, flags, _stream_handle(stream)))
        return slot

    def detectAndCompute(self, img, slot: int | None = None, stream=None):
        """SURF::detectAndCompute (SURF.hpp:57-58): keypoints (KEYPOINT_DTYPE
        records) and descriptors ([n][64] float32) on the host."""
        if slot is None:
            slot = self._next_slot
            self._next_slot = (self._next_slot + 1) % SURF_SLOTS
        self.detect_slot(img, slot, stream)
        return self.features(slot, stream)

    def match_slots(self, query_slot: int, train_slot: int, stream=None, host: bool = True):
        cap = self.max_features if self.max_features >= 0 else 64000
        out = np.zeros(cap, MATCH_DTYPE) if host else None
        n = C.c_int32(0)
        check(lib().gls_surf_match(self._h, query_slot, train_slot, None if out is None else out.ctypes.data, cap,
                                   C.byref(n) if host else None, _stream_handle(stream)))
        return out[:n.value].copy() if host else None

    def find_homography_slots(self, threshold: float = 1.0, max_iterations: int = 2000, stream=None):
        """FindHomography over the last match_slots result."""
        H = np.zeros(9, np.float32)
        cap = self.max_features if self.max_features >= 0 else 64000
        inl = np.zeros(cap, np.int32)
        n = C.c_int32(0)
        check(lib().gls_surf_find_homography(self._h, float(threshold), max_iterations,
                                             H.ctypes.data_as(C.POINTER(C.c_float)),
                                             inl.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(n),
                                             _stream_handle(stream)))
        return H.reshape(3, 3), inl[:n.value].copy()

    def register_frames(self, ref_slots, frame_slots, threshold: float = 1.0, max_iterations: int = 2000,
                        scale_to_full: bool = True, stream=None) -> np.ndarray:
        """Batched burst registration: frame_slots[f][c] matched against
        ref_slots[c]; per-frame homographies averaged over the channels
        (and scaled to full resolution), [n_frames][3][3]."""
        fs = np.ascontiguousarray(np.asarray(frame_slots, np.int32))
        rs = np.ascontiguousarray(np.asarray(ref_slots, np.int32))
        nf, nc = fs.shape
        H = np.zeros((nf, 9), np.float32)
        check(lib().gls_surf_register_frames(self._h, rs.ctypes.data_as(C.POINTER(C.c_int32)), nc,
                                             fs.ctypes.data_as(C.POINTER(C.c_int32)), nf, float(threshold),
                                             max_iterations, int(scale_to_full),
                                             H.ctypes.data_as(C.POINTER(C.c_float)), _stream_handle(stream)))
        return H.reshape(nf, 3, 3)

    def findMatches(self, query_slot: int, train_slot: int, stream=None):
        """SURF::findMatches (SURF.hpp:65-75) on two slots: (query pt,
        train pt) pairs in match order, as float32 [n][4]."""
        m = self.match_slots(query_slot, train_slot, stream)
        kq, _ = self.features(query_slot, stream)
        kt, _ = self.features(train_slot, stream)
        return np.stack([kq["x"][m["query_idx"]], kq["y"][m["query_idx"]],
                         kt["x"][m["train_idx"]], kt["y"][m["train_idx"]]], 1).astype(np.float32)

    def raw_channels(self, raw, bayer_pattern: int, black_level: float, white_level: float,
                     exposure_multiplier: float = 1.0, channels=(1, 3), outs=None, stream=None):
        """RawChannels (pyramidFusion.cpp:106-143) into CUDA tensors (or the
        given outputs); raw is a numpy uint16 array or a CUDA tensor."""
        import torch
        h, w = raw.shape
        dev = torch.device("cuda", torch.cuda.current_device())
        if outs is None:
            outs = {c: torch.empty((h // 2, w // 2), dtype=torch.float32, device=dev) for c in channels}
        views = (ImageView * 4)()
        mask = 0
        for c, t in outs.items():
            views[c] = _view(t, 1)
            mask |= 1 << c
        host = isinstance(raw, np.ndarray)
        if host:
            raw = np.ascontiguousarray(raw, np.uint16)
        check(lib().gls_raw_channels(self._h, C.c_void_p(_ptr(raw)), w, h, _row_stride(raw), bayer_pattern,
                                     float(black_level), float(white_level), float(exposure_multiplier), mask, views,
                                     HOST_IO if host else 0, _stream_handle(stream)))
        return outs


def FindHomography(ctx: SURF, pairs: np.ndarray, threshold: float = 1.0, max_iterations: int = 2000, stream=None):
    """FindHomography(matchpoints, threshold, max_iterations, &inliers)
    (Homography.hpp:26-27) for host point pairs [n][4] = (x1, y1, x2, y2)."""
    p = np.ascontiguousarray(pairs, np.float32)
    H = np.zeros(9, np.float32)
    inl = np.zeros(max(len(p), 1), np.int32)
    n = C.c_int32(0)
    check(lib().gls_find_homography(ctx.handle, p.ctypes.data_as(C.POINTER(C.c_float)), len(p), float(threshold),
                                    max_iterations, H.ctypes.data_as(C.POINTER(C.c_float)),
                                    inl.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(n), _stream_handle(stream)))
    return H.reshape(3, 3), inl[:n.value].copy()


def ScaleHomography(H, scale: float = 2.0) -> np.ndarray:
    """ScaleHomography (Homography.hpp:29-37)."""
    h = np.ascontiguousarray(np.asarray(H, np.float32).ravel())
    out = np.zeros(9, np.float32)
    check(lib().gls_scale_homography(h.ctypes.data_as(C.POINTER(C.c_float)), float(scale),
                                     out.ctypes.data_as(C.POINTER(C.c_float))))
    return out.reshape(3, 3)


class RegisterAndFuseKernel:
    """RegisterAndFuseKernel (demosaic_kernels.hpp:690-710): fused RGBA F32
    CUDA tensors, input RGBA F32/F16 CUDA tensor."""

    def __call__(self, fused, input_image, out, homography, count: int, stream=None):
        h = np.ascontiguousarray(np.asarray(homography, np.float32).ravel())
        fv, iv, ov = _view(fused, 4), _view(input_image, 4), _view(out, 4)
        check(lib().gls_register_and_fuse(C.byref(fv), C.byref(iv), C.byref(ov),
                                          h.ctypes.data_as(C.POINTER(C.c_float)), int(count), _stream_handle(stream)))
        return out


def register_image(input_image, out, homography, stream=None):
    """registerImage (SURF.metal:518-538)."""
    h = np.ascontiguousarray(np.asarray(homography, np.float32).ravel())
    iv, ov = _view(input_image, 4), _view(out, 4)
    check(lib().gls_register_image(C.byref(iv), C.byref(ov), h.ctypes.data_as(C.POINTER(C.c_float)),
                                   _stream_handle(stream)))
    return out


def fuse_pyramid(ctx: SURF, frames, homographies, out, levels: int = 5, robustness: float = 0.0, stream=None):
    """Pyramid burst fusion (gls_fuse_pyramid): frames[0] is the reference,
    frames[f] is warped by homographies[f] (reference -> frame); CUDA
    tensors (RGBA F32/F16), out RGBA F32/F16 CUDA tensor."""
    n = len(frames)
    views = (ImageView * n)(*[_view(f, 4) for f in frames])
    H = np.zeros((n, 9), np.float32)
    for f in range(1, n):
        H[f] = np.asarray(homographies[f], np.float32).ravel()
    ov = _view(out, 4)
    check(lib().gls_fuse_pyramid(ctx.handle, views, n, H.ctypes.data_as(C.POINTER(C.c_float)), levels,
                                 float(robustness), C.byref(ov), _stream_handle(stream)))
    return out
