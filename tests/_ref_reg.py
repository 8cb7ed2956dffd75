"""ctypes binding of oracle/_ref/libglsref_reg.so: the reference's own
registration code (ImageRegistration/SURF.metal, SURF.cpp, Homography.cpp,
LeastSquaresHomography.cpp over RTL) compiled for the CPU (see
oracle/ref_reg_harness.cpp). Built by `make -C oracle ref` where the
reference tree is present; the shared object travels with the repository
snapshot, so tests that need it skip only where it was never built."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from glasscamerapublic_b200 import KEYPOINT_DTYPE, MATCH_DTYPE

REF_LIB = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libglsref_reg.so"
_lib = None


def available() -> bool:
    return REF_LIB.exists()


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        L = C.CDLL(str(REF_LIB))
        fp = C.POINTER(C.c_float)
        ip = C.POINTER(C.c_int)
        vp = C.c_void_p
        L.ref_reg_set_own_math.argtypes = [C.c_int]
        L.ref_reg_set_threads.argtypes = [C.c_int]
        L.ref_reg_integral.argtypes = [fp, C.c_int, C.c_int, fp]
        L.ref_reg_detect.argtypes = [fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, vp, fp, C.c_int, ip]
        L.ref_reg_match.argtypes = [fp, C.c_int, fp, C.c_int, vp]
        L.ref_reg_find_homography.argtypes = [fp, fp, C.c_int, C.c_float, C.c_int, fp, ip, C.c_int]
        L.ref_reg_ls_homography.argtypes = [fp, fp, C.c_int, fp]
        L.ref_reg_scale_homography.argtypes = [fp, C.c_float, fp]
        L.ref_reg_fuse.argtypes = [fp, fp, C.c_int, C.c_int, fp, C.c_int, fp]
        _lib = L
    return _lib


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def own_math(on: bool):
    """Bind the reference's atan2 / hypot calls to this library's own
    functions (True) or to the C library's (False)."""
    lib().ref_reg_set_own_math(1 if on else 0)


def integral(img):
    img = _f32(img)
    h, w = img.shape
    out = np.zeros((h + 1, w + 1), np.float32)
    lib().ref_reg_integral(_fp(img), w, h, _fp(out))
    return out


def detect(img, n_octaves=4, n_layers=2, threshold=0.02, max_features=1500, capacity=70000):
    img = _f32(img)
    h, w = img.shape
    kps = np.zeros(capacity, KEYPOINT_DTYPE)
    desc = np.zeros((capacity, 64), np.float32)
    found = C.c_int(0)
    n = lib().ref_reg_detect(_fp(img), w, h, n_octaves, n_layers, threshold, max_features, kps.ctypes.data,
                             _fp(desc), capacity, C.byref(found))
    return kps[:n].copy(), desc[:n].copy(), found.value


def match(d1, d2):
    d1, d2 = _f32(d1), _f32(d2)
    out = np.zeros(len(d1), MATCH_DTYPE)
    lib().ref_reg_match(_fp(d1), len(d1), _fp(d2), len(d2), out.ctypes.data)
    return out


def find_homography(p1, p2, threshold=1.0, iterations=2000):
    p1, p2 = _f32(p1), _f32(p2)
    n = len(p1)
    H = np.zeros(9, np.float32)
    inl = np.zeros(max(n, 1), np.int32)
    k = lib().ref_reg_find_homography(_fp(p1), _fp(p2), n, threshold, iterations, _fp(H),
                                      inl.ctypes.data_as(C.POINTER(C.c_int)), len(inl))
    return H.reshape(3, 3), inl[:k].copy()


def ls_homography(p1, p2):
    p1, p2 = _f32(p1), _f32(p2)
    H = np.zeros(9, np.float32)
    rc = lib().ref_reg_ls_homography(_fp(p1), _fp(p2), len(p1), _fp(H))
    return None if rc != 0 else H.reshape(3, 3)


def scale_homography(H, scale=2.0):
    H = _f32(np.asarray(H).ravel())
    out = np.zeros(9, np.float32)
    lib().ref_reg_scale_homography(_fp(H), scale, _fp(out))
    return out.reshape(3, 3)


def fuse(fused, inp, H, count):
    fused, inp = _f32(fused), _f32(inp)
    h, w = fused.shape[:2]
    out = np.zeros_like(fused)
    lib().ref_reg_fuse(_fp(fused), _fp(inp), w, h, _fp(_f32(np.asarray(H).ravel())), count, _fp(out))
    return out
