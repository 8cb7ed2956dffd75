"""Known-answer tests of the registration oracle (CPU, no GPU).

The reference ships no tests or vectors for SURF, RANSAC or fusion; these
pin the restatement from the mathematics and from published definitions:
  * the library's own atan2f / sinf / cosf against double precision;
  * std::mt19937's published 10000th output, and the RANSAC sample sets
    against a Python restatement of the mask-and-reject map;
  * exact integral images on integer-valued input;
  * homography recovery from exact and outlier-laden correspondences;
  * identities of the registerAndFuse warp and of the matcher;
  * a blob detector check (a dark disc is found at its centre).
"""
import numpy as np
import pytest

import _oracle_reg as R
from glasscamerapublic_b200 import scene


def _ulp_err(got, ref):
    got = np.asarray(got, np.float32)
    ref64 = np.asarray(ref, np.float64)
    ulp = np.spacing(np.abs(ref64).astype(np.float32)).astype(np.float64)
    return np.abs(got.astype(np.float64) - ref64) / ulp


def test_own_atan2_within_three_ulps():
    rng = np.random.default_rng(0)
    y = (rng.standard_normal(200000) * 10 ** rng.uniform(-3, 3, 200000)).astype(np.float32)
    x = (rng.standard_normal(200000) * 10 ** rng.uniform(-3, 3, 200000)).astype(np.float32)
    got = R.math("atan2", y, x)
    ref = np.arctan2(y.astype(np.float64), x.astype(np.float64))
    assert _ulp_err(got, ref).max() <= 3.0


def test_own_atan2_special_values():
    inf = np.float32(np.inf)
    cases = [(0.0, 1.0, 0.0), (-0.0, 1.0, -0.0), (0.0, -1.0, np.pi), (-0.0, -1.0, -np.pi), (0.0, 0.0, 0.0),
             (-0.0, 0.0, -0.0), (0.0, -0.0, np.pi), (1.0, 0.0, np.pi / 2), (-1.0, 0.0, -np.pi / 2),
             (inf, inf, np.pi / 4), (inf, -inf, 3 * np.pi / 4), (1.0, inf, 0.0), (1.0, -inf, np.pi)]
    for y, x, ref in cases:
        got = R.math("atan2", np.float32(y), np.float32(x))[0]
        assert np.float32(got) == np.float32(ref) and np.signbit(got) == np.signbit(np.float32(ref)), (y, x, got)
    assert np.isnan(R.math("atan2", np.float32(np.nan), np.float32(1.0))[0])


@pytest.mark.parametrize("fn", ["sin", "cos"])
def test_own_sin_cos_within_two_ulps(fn):
    rng = np.random.default_rng(1)
    a = np.concatenate([rng.uniform(-0.06, 0.06, 50000), rng.uniform(-1000, 1000, 50000)]).astype(np.float32)
    got = R.math(fn, a)
    ref = getattr(np, fn)(a.astype(np.float64))
    assert _ulp_err(got, ref).max() <= 2.0
    small = np.abs(a) <= 0.06  # the range the descriptor rotation reaches
    assert _ulp_err(got[small], ref[small]).max() <= 0.51


def _mt19937(seed=5489):
    bg = np.random.MT19937(0)
    bg._legacy_seeding(seed)
    return bg


def test_mt19937_published_value():
    # the C++ standard requires the 10000th output of a default-constructed
    # std::mt19937 to be 4123659995
    assert int(_mt19937().random_raw(10000)[-1]) == 4123659995


@pytest.mark.parametrize("n", [4, 5, 37, 1500, 64000])
def test_ransac_samples_mask_and_reject(n):
    it = 300
    got = R.samples(it, n, sampler=0)
    bg = _mt19937()
    w = int(np.ceil(np.log2(n))) if n > 1 else 0
    mask = (1 << w) - 1
    exp = []
    for _ in range(it):
        s = set()
        while len(s) < 4:
            while True:
                u = int(bg.random_raw()) & mask
                if u < n:
                    break
            s.add(u)
        exp.append(sorted(s))
    assert np.array_equal(got, np.array(exp, np.int32))


def test_integral_exact_for_integer_values():
    rng = np.random.default_rng(2)
    img = (rng.integers(0, 16, size=(97, 131)) + 0.5).astype(np.float32)
    s = R.integral(img)
    exact = np.zeros((98, 132))
    exact[1:, 1:] = np.cumsum(np.cumsum(img - 0.5, 0), 1)
    assert np.array_equal(s.astype(np.float64), exact)
    assert np.all(s[0] == 0) and np.all(s[:, 0] == 0)


def _proj(H, p):
    q = np.c_[p, np.ones(len(p))] @ np.asarray(H, np.float64).T
    return q[:, :2] / q[:, 2:]


@pytest.mark.parametrize("n", [4, 100])
def test_ls_homography_recovers_exact_correspondences(n):
    rng = np.random.default_rng(n)
    Ht = np.array([[1.02, -0.03, 12.5], [0.025, 0.98, -7.25], [2e-5, -1e-5, 1.0]])
    p1 = rng.uniform(0, 2000, size=(n, 2)).astype(np.float32)
    p2 = _proj(Ht, p1.astype(np.float64)).astype(np.float32)
    H = R.ls_homography(p1, p2)
    assert H is not None
    assert scene.corner_error(H, Ht, 2000, 2000) < 2e-3


def test_ls_homography_degenerate_spread():
    p = np.tile(np.array([[10.0, 20.0]], np.float32), (4, 1))
    assert R.ls_homography(p, p) is None


def test_ransac_rejects_outliers():
    rng = np.random.default_rng(3)
    Ht = np.array([[0.999, 0.017, -9.0], [-0.017, 0.999, 14.0], [5e-6, -3e-6, 1.0]])
    n = 600
    p1 = rng.uniform(0, 2016, size=(n, 2))
    p2 = _proj(Ht, p1)
    bad = rng.random(n) < 0.3
    p2[bad] += rng.uniform(20, 200, size=(bad.sum(), 2)) * rng.choice([-1, 1], size=(bad.sum(), 2))
    H, inl, loss = R.find_homography(p1.astype(np.float32), p2.astype(np.float32), 1.0, 2000)
    assert scene.corner_error(H, Ht, 2016, 1512) < 0.05
    assert set(np.flatnonzero(~bad)) <= set(inl.tolist())
    assert loss == float(bad.sum())


def test_scale_homography_is_s_h_s_inverse():
    H = np.array([[1.0, 0.1, 3.0], [0.2, 1.0, -4.0], [1e-4, 2e-4, 1.0]], np.float32)
    S = np.diag([2.0, 2.0, 1.0])
    ref = (S @ H.astype(np.float64) @ np.linalg.inv(S)).astype(np.float32)
    assert np.array_equal(R.scale_homography(H), ref)


def test_fuse_identity_and_running_mean():
    rng = np.random.default_rng(4)
    a = rng.random((40, 50, 4), dtype=np.float32)
    b = rng.random((40, 50, 4), dtype=np.float32)
    I = np.eye(3, dtype=np.float32)
    assert np.array_equal(R.fuse(a, b, I, 1), b)  # count 1 replaces the fused frame
    assert np.array_equal(R.fuse(a, a, I, 2), a)
    assert np.allclose(R.fuse(a, b, I, 2), (a + b) / 2, atol=1e-7)


def test_fuse_integer_shift_is_exact():
    rng = np.random.default_rng(5)
    a = rng.random((40, 50, 4), dtype=np.float32)
    H = np.array([[1, 0, 3], [0, 1, -2], [0, 0, 1]], np.float32)
    out = R.fuse(np.zeros_like(a), a, H, 1)
    assert np.array_equal(out[2:, :47], a[:-2, 3:])


def test_raw_channel_tone_curve():
    rng = np.random.default_rng(6)
    raw = rng.integers(0, 4096, size=(64, 80)).astype(np.uint16)
    out = R.raw_channel(raw, 2, 1, 512.0, 4095.0, 1.0)
    v = raw[0::2, 1::2].astype(np.float64)  # G of RGGB at (1, 0)
    x = np.clip((v - 512.0) / 4095.0, 0, 1)

    def sig(t, s=3.5):
        return 0.5 * (np.tanh(s * t - 0.3 * s) + 1)

    ref = (sig(np.sqrt(0.95 * x)) - sig(0.0)) / (sig(1.0) - sig(0.0))
    assert np.abs(out - ref).max() < 2e-6


def test_detector_finds_a_blob_at_its_centre():
    h, w = 256, 256
    yy, xx = np.mgrid[0:h, 0:w]
    img = np.full((h, w), 0.8, np.float32)
    cx, cy, r = 121.0, 133.0, 6.0
    img[(xx - cx) ** 2 + (yy - cy) ** 2 <= r * r] = 0.1
    kps, desc, _ = R.detect(img, max_features=-1)
    d = np.hypot(kps["x"] - cx, kps["y"] - cy)
    assert d.min() < 1.0
    k = kps[np.argmin(d)]
    assert k["class_id"] == 1  # dark blob: positive Hessian trace
    assert np.all(np.abs(kps["angle"]) <= np.pi + 1e-6)
    assert np.allclose(np.linalg.norm(desc, axis=1)[kps["size"] > 0], 1.0, atol=1e-5)


def test_matcher_matches_identical_descriptors_to_themselves():
    rng = np.random.default_rng(7)
    d = rng.standard_normal((50, 64)).astype(np.float32)
    m = R.match(d, d)
    assert np.all(m["distance"] == 0)
    assert np.array_equal(np.sort(m["query_idx"]), np.arange(50))
    assert np.all(m["query_idx"] == m["train_idx"])
    assert np.all(np.diff(m["query_idx"]) > 0)  # equal distances: query order
