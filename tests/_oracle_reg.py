"""ctypes binding of the registration oracle (oracle/gls_oracle_reg.hpp,
built into oracle/liboracle.so) for the tests: RawChannels, the SURF
integral / detector / descriptor / matcher, RANSAC + least-squares
homography and the registerAndFuse warp."""
from __future__ import annotations

import ctypes as C

import numpy as np

import _oracle
from glasscamerapublic_b200 import KEYPOINT_DTYPE, MATCH_DTYPE

_done = False


def lib() -> C.CDLL:
    global _done
    L = _oracle.lib()
    if not _done:
        fp = C.POINTER(C.c_float)
        ip = C.POINTER(C.c_int)
        vp = C.c_void_p
        L.orc_reg_math.argtypes = [C.c_int, fp, fp, fp, C.c_int]
        L.orc_reg_raw_channel.argtypes = [vp, C.c_int, C.c_int, C.c_size_t, C.c_int, C.c_int, C.c_float, C.c_float,
                                          C.c_float, fp]
        L.orc_reg_integral.argtypes = [fp, C.c_int, C.c_int, fp]
        L.orc_reg_detect.argtypes = [fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, vp, fp, C.c_int, ip,
                                     C.c_int]
        L.orc_reg_describe.argtypes = [fp, C.c_int, C.c_int, vp, C.c_int, fp]
        L.orc_reg_match.argtypes = [fp, C.c_int, fp, C.c_int, vp]
        L.orc_reg_ls_homography.argtypes = [fp, fp, C.c_int, fp]
        L.orc_reg_samples.argtypes = [C.c_int, C.c_int, C.c_int, ip]
        L.orc_reg_find_homography.argtypes = [fp, fp, C.c_int, C.c_float, C.c_int, C.c_int, fp, ip, ip, fp]
        L.orc_reg_scale_homography.argtypes = [fp, fp]
        L.orc_reg_fuse.argtypes = [fp, fp, C.c_int, C.c_int, fp, C.c_int, fp]
        _done = True
    return L


def _fp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))


def _ip(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_int))


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def math(fn: str, a, b=None):
    a = _f32(np.atleast_1d(a))
    b = _f32(np.atleast_1d(b)) if b is not None else a
    out = np.zeros_like(a)
    lib().orc_reg_math({"atan2": 0, "sin": 1, "cos": 2}[fn], _fp(a), _fp(b), _fp(out), a.size)
    return out


def raw_channel(raw, pattern, c, black, white, exposure=1.0):
    raw = np.ascontiguousarray(raw, np.uint16)
    h, w = raw.shape
    out = np.zeros((h // 2, w // 2), np.float32)
    assert lib().orc_reg_raw_channel(raw.ctypes.data, w, h, w, pattern, c, black, white, exposure, _fp(out)) == 0
    return out


def integral(img):
    img = _f32(img)
    h, w = img.shape
    out = np.zeros((h + 1, w + 1), np.float32)
    lib().orc_reg_integral(_fp(img), w, h, _fp(out))
    return out


def detect(img, n_octaves=4, n_layers=2, threshold=0.02, max_features=1500, capacity=70000, per_axis=False):
    img = _f32(img)
    h, w = img.shape
    kps = np.zeros(capacity, KEYPOINT_DTYPE)
    desc = np.zeros((capacity, 64), np.float32)
    found = C.c_int(0)
    n = lib().orc_reg_detect(_fp(img), w, h, n_octaves, n_layers, threshold, max_features, kps.ctypes.data,
                             _fp(desc), capacity, C.byref(found), 1 if per_axis else 0)
    return kps[:n].copy(), desc[:n].copy(), found.value


def describe(img, kps):
    img = _f32(img)
    h, w = img.shape
    k = np.ascontiguousarray(kps.copy())
    desc = np.zeros((len(k), 64), np.float32)
    lib().orc_reg_describe(_fp(img), w, h, k.ctypes.data, len(k), _fp(desc))
    return k, desc


def match(d1, d2):
    d1, d2 = _f32(d1), _f32(d2)
    out = np.zeros(len(d1), MATCH_DTYPE)
    lib().orc_reg_match(_fp(d1), len(d1), _fp(d2), len(d2), out.ctypes.data)
    return out


def ls_homography(p1, p2):
    p1, p2 = _f32(p1), _f32(p2)
    H = np.zeros(9, np.float32)
    rc = lib().orc_reg_ls_homography(_fp(p1), _fp(p2), len(p1), _fp(H))
    return None if rc != 0 else H.reshape(3, 3)


def samples(iterations, n, sampler=0):
    out = np.zeros((iterations, 4), np.int32)
    lib().orc_reg_samples(iterations, n, sampler, _ip(out))
    return out


def find_homography(p1, p2, threshold=1.0, iterations=2000, sampler=0):
    p1, p2 = _f32(p1), _f32(p2)
    n = len(p1)
    H = np.zeros(9, np.float32)
    inl = np.zeros(max(n, 1), np.int32)
    ni = C.c_int(0)
    loss = C.c_float(0)
    assert lib().orc_reg_find_homography(_fp(p1), _fp(p2), n, threshold, iterations, sampler, _fp(H), _ip(inl),
                                         C.byref(ni), C.byref(loss)) == 0
    return H.reshape(3, 3), inl[:ni.value].copy(), loss.value


def scale_homography(H):
    H = _f32(np.asarray(H).ravel())
    out = np.zeros(9, np.float32)
    lib().orc_reg_scale_homography(_fp(H), _fp(out))
    return out.reshape(3, 3)


def fuse(fused, inp, H, count):
    fused, inp = _f32(fused), _f32(inp)
    h, w = fused.shape[:2]
    out = np.zeros_like(fused)
    lib().orc_reg_fuse(_fp(fused), _fp(inp), w, h, _fp(_f32(np.asarray(H).ravel())), count, _fp(out))
    return out
