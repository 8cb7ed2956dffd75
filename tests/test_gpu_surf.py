"""GPU parity of the registration and fusion path against the CPU oracle
(oracle/gls_oracle_reg.hpp), through the C ABI.

Every stage is bit-exact: the library and the oracle evaluate the same
float expressions with one rounding per operation and share the library's
own atan2f / sinf / cosf, so integral images, keypoints, descriptors,
matches, homographies and warped pixels must be identical.
"""
import ctypes as C

import numpy as np
import pytest

import _oracle_reg as R
import glasscamerapublic_b200 as g
from glasscamerapublic_b200 import scene
from glasscamerapublic_b200.registration import (SURF, FindHomography, RegisterAndFuseKernel, ScaleHomography,
                                                 register_image)

pytestmark = pytest.mark.gpu


def _gray(w=512, h=384, seed=3, pattern=2):
    wl = scene.Workload("reg", w * 2, h * 2, gain=1.5, read=4.0, iso=800, seed=seed, pattern=pattern)
    raw, _ = scene.make_raw(wl)
    return raw, R.raw_channel(raw, pattern, 1, 512.0, 4095.0)


def _integral(surf):
    v = g.ImageView()
    g.check(g.lib().gls_surf_plane(surf.handle, g.SURF_PLANE_INTEGRAL, C.byref(v)))
    out = np.zeros((v.height, v.width), np.float32)
    dst = g.ImageView(C.c_void_p(out.ctypes.data), v.width, v.height, 1, g.F32, out.strides[0])
    g.check(g.lib().gls_copy_view(C.byref(v), C.byref(dst), 0, None))  # device to host, synchronous
    return out


@pytest.mark.parametrize("pattern", [0, 2])
def test_raw_channels_bit_exact(pattern):
    import torch
    wl = scene.Workload("reg", 640, 480, gain=1.5, read=4.0, iso=800, seed=5, pattern=pattern)
    raw, _ = scene.make_raw(wl)
    s = SURF(320, 240)
    try:
        outs = s.raw_channels(raw, pattern, 512.0, 4095.0, 1.25, channels=(0, 1, 2, 3))
        torch.cuda.synchronize()
        for c in range(4):
            ref = R.raw_channel(raw, pattern, c, 512.0, 4095.0, 1.25)
            assert np.array_equal(outs[c].cpu().numpy(), ref), c
        # device input gives the same planes
        outs2 = s.raw_channels(torch.from_numpy(raw.astype(np.int16)).cuda(), pattern, 512.0, 4095.0, 1.25,
                               channels=(1,))
        torch.cuda.synchronize()
        assert np.array_equal(outs2[1].cpu().numpy(), R.raw_channel(raw, pattern, 1, 512.0, 4095.0, 1.25))
    finally:
        s.close()


@pytest.mark.parametrize("size", [(512, 384), (333, 257)])
def test_integral_bit_exact(size):
    w, h = size
    rng = np.random.default_rng(1)
    img = rng.random((h, w), dtype=np.float32)
    s = SURF(w, h, max_features=100)
    try:
        s.detectAndCompute(img, slot=0)
        assert np.array_equal(_integral(s), R.integral(img))
    finally:
        s.close()


def test_integral_exact_for_integers():
    # v - 0.5 integer-valued: the float prefix sums are exact integers
    rng = np.random.default_rng(2)
    w, h = 200, 150
    img = (rng.integers(0, 8, size=(h, w)) + 0.5).astype(np.float32)
    s = SURF(w, h, max_features=10)
    try:
        s.detectAndCompute(img, slot=0)
        exact = np.zeros((h + 1, w + 1), np.float64)
        exact[1:, 1:] = np.cumsum(np.cumsum(img.astype(np.float64) - 0.5, 0), 1)
        assert np.array_equal(_integral(s).astype(np.float64), exact)
    finally:
        s.close()


@pytest.mark.parametrize("max_features,seed", [(1500, 3), (-1, 4), (20, 5)])
def test_detect_and_compute_bit_exact(max_features, seed):
    raw, img = _gray(seed=seed)
    h, w = img.shape
    s = SURF(w, h, max_features=max_features)
    try:
        kps, desc = s.detectAndCompute(img, slot=1)
        rk, rd, found = R.detect(img, max_features=max_features)
        assert len(kps) == len(rk) and len(rk) > 0, (len(kps), len(rk), found)
        for f in rk.dtype.names:
            assert np.array_equal(kps[f], rk[f]), f
        assert np.array_equal(desc, rd)
    finally:
        s.close()


def test_reference_detector_leaves_the_undescribed_tail():
    # 45 keypoints: the reference's SURFInvoker::run describes the first 36
    raw, img = _gray(seed=3)
    h, w = img.shape
    s = SURF(w, h, max_features=-1)
    try:
        kps, desc = s.detectAndCompute(img, slot=0)
        assert len(kps) == 45
        assert np.all(kps["angle"][36:] == -1) and not np.any(desc[36:])
        assert np.all(kps["angle"][:36] != -1)
    finally:
        s.close()


@pytest.mark.parametrize("seed", [3, 4])
def test_corrected_detector_bit_exact(seed):
    raw, img = _gray(seed=seed)
    h, w = img.shape
    s = SURF(w, h, max_features=-1, corrected=True)
    try:
        kps, desc = s.detectAndCompute(img, slot=0)
        rk, rd, _ = R.detect(img, max_features=-1, per_axis=True)
        assert len(kps) == len(rk) > 0
        for f in rk.dtype.names:
            assert np.array_equal(kps[f], rk[f]), f
        assert np.array_equal(desc, rd)
        assert np.all(kps["angle"] != -1)
    finally:
        s.close()


def test_detect_device_input_matches_host_input():
    import torch
    raw, img = _gray(seed=6)
    h, w = img.shape
    s = SURF(w, h, max_features=1500)
    try:
        k1, d1 = s.detectAndCompute(img, slot=0)
        k2, d2 = s.detectAndCompute(torch.from_numpy(img).cuda(), slot=1)
        assert np.array_equal(k1, k2) and np.array_equal(d1, d2)
    finally:
        s.close()


def test_match_and_homography_bit_exact():
    wl = scene.Workload("reg", 1024, 768, gain=1.5, read=4.0, iso=800, seed=3000)
    raws, _, Hs = scene.make_burst(wl, 2)
    a = R.raw_channel(raws[0], 2, 1, 512.0, 4095.0)
    b = R.raw_channel(raws[1], 2, 1, 512.0, 4095.0)
    h, w = a.shape
    s = SURF(w, h, max_features=1500)
    try:
        s.detectAndCompute(a, slot=0)
        s.detectAndCompute(b, slot=1)
        m = s.match_slots(0, 1)
        k1, d1, _ = R.detect(a)
        k2, d2, _ = R.detect(b)
        rm = R.match(d1, d2)
        assert np.array_equal(m, rm)
        H, inl = s.find_homography_slots(1.0, 2000)
        p1 = np.stack([k1["x"][rm["query_idx"]], k1["y"][rm["query_idx"]]], 1)
        p2 = np.stack([k2["x"][rm["train_idx"]], k2["y"][rm["train_idx"]]], 1)
        rH, rinl, _ = R.find_homography(p1, p2, 1.0, 2000, sampler=0)
        assert np.array_equal(H, rH)
        assert np.array_equal(inl, rinl)
    finally:
        s.close()


@pytest.mark.parametrize("outliers", [0.0, 0.3])
def test_find_homography_host_pairs(outliers):
    rng = np.random.default_rng(7)
    Ht = np.array([[1.01, 0.02, 5.0], [-0.015, 0.99, -3.0], [1e-5, -2e-5, 1.0]])
    n = 400
    p1 = rng.uniform(0, 1000, size=(n, 2))
    q = np.c_[p1, np.ones(n)] @ Ht.T
    p2 = q[:, :2] / q[:, 2:]
    bad = rng.random(n) < outliers
    p2[bad] += rng.uniform(-80, 80, size=(bad.sum(), 2))
    pairs = np.c_[p1, p2].astype(np.float32)
    s = SURF(64, 64, max_features=10)
    try:
        H, inl = FindHomography(s, pairs, 1.0, 500)
        rH, rinl, _ = R.find_homography(pairs[:, :2], pairs[:, 2:], 1.0, 500, sampler=0)
        assert np.array_equal(H, rH) and np.array_equal(inl, rinl)
        assert scene.corner_error(H, Ht, 1000, 1000) < 0.1
        assert set(np.flatnonzero(~bad)) <= set(inl.tolist()) | set(np.flatnonzero(bad))
    finally:
        s.close()


def test_scale_homography_matches_reference_form():
    H = np.array([[1.0, 0.1, 3.0], [0.2, 1.0, -4.0], [1e-4, 2e-4, 1.0]], np.float32)
    assert np.array_equal(ScaleHomography(H, 7.0), R.scale_homography(H))


@pytest.mark.parametrize("count", [1, 2, 3])
@pytest.mark.parametrize("f16", [False, True])
def test_register_and_fuse_bit_exact(count, f16):
    import torch
    rng = np.random.default_rng(count)
    h, w = 96, 128
    fused = rng.random((h, w, 4), dtype=np.float32)
    inp = rng.random((h, w, 4), dtype=np.float32)
    if f16:
        inp = inp.astype(np.float16).astype(np.float32)
    H = np.array([[0.999, 0.01, 2.5], [-0.012, 1.001, -1.25], [1e-5, -2e-5, 1.0]], np.float32)
    ref = R.fuse(fused, inp, H, count)
    tf = torch.from_numpy(fused).cuda()
    ti = torch.from_numpy(inp).cuda().half() if f16 else torch.from_numpy(inp).cuda()
    out = torch.empty_like(tf)
    RegisterAndFuseKernel()(tf, ti, out, H, count)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), ref)
    # in place, as the reference calls it (fused and out the same texture)
    RegisterAndFuseKernel()(tf, ti, tf, H, count)
    torch.cuda.synchronize()
    assert np.array_equal(tf.cpu().numpy(), ref)


def test_register_image_identity_is_copy():
    import torch
    rng = np.random.default_rng(9)
    img = torch.from_numpy(rng.random((64, 80, 4), dtype=np.float32)).cuda()
    out = torch.empty_like(img)
    register_image(img, out, np.eye(3))
    torch.cuda.synchronize()
    assert torch.equal(out, img)


@pytest.mark.parametrize("corrected,bound", [(False, 2.5), (True, 1.0)])
def test_burst_registration_recovers_warps(corrected, bound):
    # RawChannels (G, G2) -> SURF -> match -> RANSAC per channel, running
    # average, ScaleHomography: the main() driver of pyramidFusion.cpp:276-346.
    # The reference's detector moves keypoints by the scale offset along x
    # and y as well (SURF.metal:200), which costs it sub-pixel accuracy; the
    # corrected detector registers these frames to well under a pixel.
    wl = scene.Workload("burst", 2048, 1536, gain=1.5, read=4.0, iso=800, seed=3001)
    raws, _, Hs = scene.make_burst(wl, 3)
    s = SURF(1024, 768, max_features=1500, corrected=corrected)
    try:
        ref = s.raw_channels(raws[0], 2, 512.0, 4095.0)
        s.detect_slot(ref[1], 0)
        s.detect_slot(ref[3], 1)
        for i in (1, 2):
            ch = s.raw_channels(raws[i], 2, 512.0, 4095.0)
            Hacc = np.zeros((3, 3), np.float32)
            for c, (slot_ref, plane) in enumerate(((0, ch[1]), (1, ch[3]))):
                s.detect_slot(plane, 2 + c)
                s.match_slots(slot_ref, 2 + c, host=False)
                Hc, _ = s.find_homography_slots(1.0, 2000)
                Hacc = (Hc + Hacc * np.float32(c)) / np.float32(c + 1)
            Hf = ScaleHomography(Hacc, 2)
            err = scene.corner_error(Hf, Hs[i], wl.width, wl.height)
            assert err < bound, (i, err)
    finally:
        s.close()


def test_register_frames_batch_equals_single_jobs():
    # the batched burst registration gives the per-job results bit for bit
    wl = scene.Workload("burst", 1024, 768, gain=1.5, read=4.0, iso=800, seed=3002)
    raws, _, Hs = scene.make_burst(wl, 4)
    s = SURF(512, 384, max_features=1500, corrected=True)
    try:
        planes = []
        for f, r in enumerate(raws):
            ch = s.raw_channels(r, 2, 512.0, 4095.0)
            s.detect_slot(ch[1], 2 * f)
            s.detect_slot(ch[3], 2 * f + 1)
            planes.append(ch)
        Hb = s.register_frames([0, 1], [[2 * f, 2 * f + 1] for f in range(1, 4)], 1.0, 2000, True)
        for f in range(1, 4):
            acc = np.zeros((3, 3), np.float32)
            for c in range(2):
                s.match_slots(c, 2 * f + c, host=False)
                Hc, _ = s.find_homography_slots(1.0, 2000)
                acc = (Hc + acc * np.float32(c)) / np.float32(c + 1)
            assert np.array_equal(Hb[f - 1], ScaleHomography(acc, 2)), f
            assert scene.corner_error(Hb[f - 1], Hs[f], 1024, 768) < 1.0
    finally:
        s.close()
