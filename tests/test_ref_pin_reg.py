"""The registration oracle (oracle/gls_oracle_reg.hpp) pinned against the
reference's own registration code compiled for the CPU
(oracle/_ref/libglsref_reg.so, see oracle/ref_reg_harness.cpp): SURF.metal's
integral, Hessian, maxima, matching and fusion kernels, SURF.cpp's
orientation and descriptor code, Homography.cpp's RANSAC over RTL and
LeastSquaresHomography.cpp's Jacobi least squares.

With the reference's atan2 / hypot calls bound to the library's own
functions (own_math), every stage is bit-exact. With the C library's, the
keypoint angles move by at most 2 float ulps; nothing else changes.
RANSAC is compared with the oracle's libstdc++ sampler (sampler=1): the
reference draws through std::uniform_int_distribution, whose mapping is the
standard library's (the library itself uses libc++'s, the one Apple's
toolchain builds the reference with)."""
import numpy as np
import pytest

import _oracle_reg as R
import _ref_reg as F
from glasscamerapublic_b200 import scene

pytestmark = pytest.mark.skipif(not F.available(), reason="oracle/_ref/libglsref_reg.so not built")


@pytest.fixture
def own_math():
    F.own_math(True)
    yield
    F.own_math(False)


@pytest.fixture(scope="module")
def burst():
    wl = scene.Workload("reg", 1024, 768, gain=1.5, read=4.0, iso=800, seed=3000)
    raws, _, Hs = scene.make_burst(wl, 2)
    return [R.raw_channel(r, 2, 1, 512.0, 4095.0) for r in raws], Hs


@pytest.mark.parametrize("size", [(512, 384), (64, 48), (8, 8)])
def test_integral_bit_exact(size):
    w, h = size
    img = np.random.default_rng(w).random((h, w), dtype=np.float32)
    assert np.array_equal(F.integral(img), R.integral(img))


@pytest.mark.parametrize("size", [(131, 97), (131, 96), (128, 97)])
def test_integral_ragged_sizes(size):
    # the reference's kernels run a short last threadgroup where the width or
    # the height is not a multiple of 8 and leave some entries unwritten
    # (NaN here, stale texture memory on the device): every entry they do
    # write equals the oracle's, and the unwritten ones are exactly those of
    # the short groups
    w, h = size
    img = np.random.default_rng(h).random((h, w), dtype=np.float32)
    ref, orc = F.integral(img), R.integral(img)
    wrote = ~np.isnan(ref)
    assert np.array_equal(ref[wrote], orc[wrote])
    expect = np.zeros_like(wrote)
    r = np.arange(h + 1)[:, None]
    c = np.arange(w + 1)[None, :]
    if w % 8:  # column pass: group (w // 8) has w % 8 threads; thread t stores image row y + t
        expect |= (c >= 8 * (w // 8) + 1) & (r >= 1) & (((r - 1) % 8) >= w % 8)
    if h % 8:  # row pass: thread t stores sum column y + t of the last rows
        expect |= (r >= 8 * (h // 8) + 1) & (c >= 1) & (((c - 1) % 8) >= h % 8)
    assert np.array_equal(~wrote, expect)


def _raw_gray(w, h, seed):
    wl = scene.Workload("reg", 2 * w, 2 * h, gain=1.5, read=4.0, iso=800, seed=seed)
    raw, _ = scene.make_raw(wl)
    return R.raw_channel(raw, 2, 1, 512.0, 4095.0)


@pytest.mark.parametrize("max_features", [-1, 1500, 40])
def test_detect_and_compute_bit_exact(own_math, max_features):
    # 512 x 384 at seed 3 has 45 keypoints: more than 32 and fewer than 57,
    # so the reference's SURFInvoker::run leaves the last 9 undescribed
    img = _raw_gray(512, 384, 3)
    rk, rd, rf = F.detect(img, max_features=max_features)
    ok, od, of = R.detect(img, max_features=max_features)
    assert rf == of and len(rk) == len(ok) > 0
    for f in rk.dtype.names:
        assert np.array_equal(rk[f], ok[f]), f
    assert np.array_equal(rd, od)
    if max_features == -1:
        assert len(rk) == 45 and np.all(rk["angle"][36:] == -1) and not np.any(rd[36:])


def test_detect_and_compute_libm_angles_within_two_ulps(burst):
    img = burst[0][0]
    rk, rd, _ = F.detect(img)
    ok, od, _ = R.detect(img)
    for f in rk.dtype.names:
        if f != "angle":
            assert np.array_equal(rk[f], ok[f]), f
    ulp = np.spacing(np.abs(ok["angle"]).astype(np.float32))
    assert np.all(np.abs(rk["angle"] - ok["angle"]) <= 2 * ulp)
    assert np.allclose(rd, od, rtol=0, atol=1e-6)


def test_match_and_homography_bit_exact(own_math, burst):
    (a, b), Hs = burst
    k1, d1, _ = F.detect(a)
    k2, d2, _ = F.detect(b)
    m = F.match(d1, d2)
    assert np.array_equal(m, R.match(d1, d2))
    p1 = np.stack([k1["x"][m["query_idx"]], k1["y"][m["query_idx"]]], 1)
    p2 = np.stack([k2["x"][m["train_idx"]], k2["y"][m["train_idx"]]], 1)
    H, inl = F.find_homography(p1, p2, 1.0, 2000)
    oH, oinl, _ = R.find_homography(p1, p2, 1.0, 2000, sampler=1)
    assert np.array_equal(H, oH) and np.array_equal(inl, oinl)
    assert scene.corner_error(R.scale_homography(H), Hs[1], 1024, 768) < 1.0


@pytest.mark.parametrize("n,outliers", [(4, 0.0), (60, 0.0), (300, 0.25)])
def test_least_squares_and_ransac(own_math, n, outliers):
    rng = np.random.default_rng(n)
    Ht = np.array([[1.01, 0.02, 5.0], [-0.015, 0.99, -3.0], [1e-5, -2e-5, 1.0]])
    p1 = rng.uniform(0, 1000, size=(n, 2))
    q = np.c_[p1, np.ones(n)] @ Ht.T
    p2 = q[:, :2] / q[:, 2:]
    bad = rng.random(n) < outliers
    p2[bad] += rng.uniform(-80, 80, size=(bad.sum(), 2))
    p1, p2 = p1.astype(np.float32), p2.astype(np.float32)
    assert np.array_equal(F.ls_homography(p1, p2), R.ls_homography(p1, p2))
    H, inl = F.find_homography(p1, p2, 1.0, 500)
    oH, oinl, _ = R.find_homography(p1, p2, 1.0, 500, sampler=1)
    assert np.array_equal(H, oH) and np.array_equal(inl, oinl)


def test_least_squares_degenerate_spread():
    p = np.tile(np.array([[10.0, 20.0]], np.float32), (4, 1))
    assert F.ls_homography(p, p) is None and R.ls_homography(p, p) is None


def test_scale_homography_bit_exact():
    H = np.array([[1.0, 0.1, 3.0], [0.2, 1.0, -4.0], [1e-4, 2e-4, 1.0]], np.float32)
    for scale in (2.0, 7.0):  # the reference scales by 2 whatever the argument
        assert np.array_equal(F.scale_homography(H, scale), R.scale_homography(H))


@pytest.mark.parametrize("count", [1, 2, 3])
def test_register_and_fuse(count):
    # the reference samples at ((x + 0.5) / w) * w - 0.5, a round trip the
    # texture unit makes in its own fixed-point precision; the library
    # samples at x itself, so the two agree to float rounding of the weights
    rng = np.random.default_rng(count)
    fused = rng.random((96, 128, 4), dtype=np.float32)
    inp = rng.random((96, 128, 4), dtype=np.float32)
    H = np.array([[0.999, 0.01, 2.5], [-0.012, 1.001, -1.25], [1e-5, -2e-5, 1.0]], np.float32)
    assert np.allclose(F.fuse(fused, inp, H, count), R.fuse(fused, inp, H, count), rtol=0, atol=2e-5)
    eye = np.eye(3, dtype=np.float32)  # the round trip moves even an identity warp off the texel centres
    assert np.allclose(F.fuse(fused, inp, eye, count), R.fuse(fused, inp, eye, count), rtol=0, atol=2e-5)
