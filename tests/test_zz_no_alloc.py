"""gls_pca_basis_noalloc: the PCA basis of an image computed with no device
allocation, for callers that cannot call cudaMalloc where they need it (a
real-time capture thread that must not block in the allocator, or an
application whose device memory is all owned by another allocator). Its
scratch is a fixed array inside the library; the caller passes only the
input image and the output basis.

The check: through the C ABI, two calls in a row (and a third after a
different image, since every call reuses the same array) give the basis
that the converter's own path (gls_pyramid_denoise + gls_converter_pca_basis)
gives for the same image, within 1e-5 per entry; an image beyond the
array's capacity is rejected.

This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

import glasscamerapublic_b200 as g
from glasscamerapublic_b200 import scene

pytestmark = pytest.mark.gpu


def _image(w, h, seed):
    rng = np.random.default_rng(seed)
    img = np.zeros((h, w, 4), np.float32)
    clean = scene.clean_scene(w, h, seed)
    img[..., 0] = 0.1 + 0.9 * clean[..., 1] + 0.01 * rng.standard_normal((h, w))
    img[..., 1] = 0.05 * rng.standard_normal((h, w))
    img[..., 2] = 0.05 * rng.standard_normal((h, w))
    return img


def _converter_basis(conv, img):
    """Basis from the converter's path: a 1-level pyramid denoise of img."""
    wl = scene.Workload("z", img.shape[1], img.shape[0], levels=1, seed=1)
    p = scene.make_params(wl)
    p.levels = 1
    grad = np.zeros(img.shape[:2] + (2,), np.float32)
    g.PyramidProcessor(conv).denoise(img, grad, p)
    return conv.pca_basis(0)


def _noalloc_basis(img_dev, out_dev, stream):
    h, w = img_dev.shape[:2]
    dt = g.F16 if img_dev.dtype == __import__("torch").float16 else g.F32
    v = g.ImageView(C.c_void_p(img_dev.data_ptr()), w, h, 4, dt, img_dev.stride(0) * img_dev.element_size())
    g.check(g.lib().gls_pca_basis_noalloc(C.byref(v), C.c_void_p(out_dev.data_ptr()), C.c_void_p(stream.cuda_stream)))
    stream.synchronize()
    return out_dev.cpu().numpy().reshape(25, 8).copy()


def test_noalloc_basis_matches_converter_basis_on_repeated_calls():
    import torch
    conv = g.RawConverter(0)
    try:
        a = _image(640, 480, 3)
        b = _image(512, 384, 4)
        ref_a = _converter_basis(conv, a)
        ref_b = _converter_basis(conv, b)
    finally:
        conv.close()
    s = torch.cuda.Stream()
    da = torch.from_numpy(a).cuda()
    db = torch.from_numpy(b).cuda()
    out = torch.full((200,), float("nan"), dtype=torch.float32, device="cuda")
    first = _noalloc_basis(da, out, s)
    second = _noalloc_basis(da, out, s)
    assert np.allclose(first, ref_a, atol=1e-5)
    assert np.allclose(second, ref_a, atol=1e-5)
    other = _noalloc_basis(db, out, s)
    assert np.allclose(other, ref_b, atol=1e-5)
    again = _noalloc_basis(da, out, s)
    assert np.allclose(again, ref_a, atol=1e-5)
    # FP16 input gives the basis of the half-rounded image
    dh = torch.from_numpy(a.astype(np.float16)).cuda()
    half = _noalloc_basis(dh, out, s)
    assert np.allclose(half @ half.T, ref_a @ ref_a.T, atol=1e-3)


def test_noalloc_rejects_images_beyond_its_scratch():
    import torch
    # 4096 x 4112 has 512 x 514 = 263,168 patches > 262,144
    big = torch.zeros((4112, 4096, 4), dtype=torch.float16, device="cuda")
    out = torch.zeros((200,), dtype=torch.float32, device="cuda")
    v = g.ImageView(C.c_void_p(big.data_ptr()), 4096, 4112, 4, g.F16, 4096 * 8)
    rc = g.lib().gls_pca_basis_noalloc(C.byref(v), C.c_void_p(out.data_ptr()), None)
    assert rc == g.GLS_ERR_INVALID_ARG
    assert b"262144" in g.lib().gls_last_error_message()
