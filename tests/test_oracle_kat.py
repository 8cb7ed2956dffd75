"""Known-answer tests that pin the CPU oracle (no GPU).

The reference ships no tests or golden vectors for this path, so the oracle
is pinned by properties its algorithms must satisfy exactly, plus the
golden fixtures in tests/golden (see test_golden.py).
"""
import math

import numpy as np
import pytest

import _oracle as O
from glasscamerapublic_b200 import scene


def test_gaussian_taps_fold_the_gaussian():
    # gaussianKernelBilinearWeights (demosaic_utils.cpp:987-1006): the folded
    # taps carry the full Gaussian mass, and each 2x2 group's offsets are the
    # weighted centroid of its pixels (except the reference's last-tap quirk).
    for radius, n in ((1.5, 4), (4.5, 25)):
        t = O.gaussian_taps(radius)
        assert t.shape == (n, 3)
        ks = max(int(math.ceil(2 * radius)), 2)
        ks += (ks % 2 == 0)
        h = ks // 2
        g = [math.exp(-(x * x + y * y) / (2 * radius * radius)) for y in range(-h, h + 1) for x in range(-h, h + 1)]
        assert t[:, 0].sum() == pytest.approx(sum(g), rel=1e-6)
        # last tap offset quirk: width / 2.0 instead of width / 2
        assert t[-1, 1] == pytest.approx(ks / 2.0) and t[-1, 2] == pytest.approx(ks / 2.0)
        # first tap's x offset lies between the first two columns
        assert -h <= t[0, 1] <= -h + 1


def test_cam_ycbcr_inverse_roundtrip():
    f, i = O.cam_ycbcr(np.eye(3), scene.XYZ_SRGB)
    assert np.allclose(f @ i, np.eye(3), atol=1e-6)
    # luma row = the Y row of xyz_rgb for an identity camera matrix
    assert np.allclose(f[0], np.array(scene.XYZ_SRGB[3:6], np.float32))


@pytest.mark.parametrize("pattern", [0, 1, 2, 3])
def test_bayer_quad_roundtrip_is_identity(pattern):
    rng = np.random.default_rng(pattern)
    raw = rng.random((12, 18)).astype(np.float32)
    q, back = O.bayer_roundtrip(raw, pattern)
    assert np.array_equal(back, raw)
    # the R channel of the quad image sits at the pattern's red offset
    ox, oy = scene.BAYER_OFFSETS[pattern][0]
    assert np.array_equal(q[..., 0], raw[oy::2, ox::2])


def test_downsample_constant_and_box():
    img = np.full((16, 20, 4), 0.37, np.float32)
    d = O.downsample(img, 10, 8)
    assert np.allclose(d[..., :3], 0.37, atol=1e-7)
    # exact halving = 4x4 box (1/16 weights) centred on the 2x2 block
    rng = np.random.default_rng(0)
    img = rng.random((16, 16, 4)).astype(np.float32)
    d = O.downsample(img, 8, 8)
    x, y = 3, 4
    box = img[2 * y - 1:2 * y + 3, 2 * x - 1:2 * x + 3, :3].mean(axis=(0, 1))
    assert np.allclose(d[y, x, :3], box, atol=1e-6)


def test_jacobi_matches_numpy_eigh():
    rng = np.random.default_rng(1)
    a = rng.standard_normal((25, 25))
    a = a @ a.T
    ev, vec = O.jacobi(a)
    ref = np.sort(np.linalg.eigvalsh(a))[::-1]
    assert np.allclose(ev, ref, rtol=1e-10, atol=1e-10)
    assert np.allclose(a @ vec, vec * ev, atol=1e-8)


def _numpy_pca_basis(img4):
    h, w = img4.shape[:2]
    pts = []
    for y in range(h // 8):
        for x in range(w // 8):
            ys = np.clip(np.arange(8 * y - 2, 8 * y + 3), 0, h - 1)
            xs = np.clip(np.arange(8 * x - 2, 8 * x + 3), 0, w - 1)
            pts.append(img4[np.ix_(ys, xs)][..., 0].ravel())
    cov = np.cov(np.array(pts, np.float64), rowvar=False)
    ev, vec = np.linalg.eigh(cov)
    return ev[::-1], vec[:, ::-1]


def test_pca_basis_matches_numpy_covariance_eigh():
    # collectPatches + build_pca_space (demosaic.metal:755-772, PCA.cpp:23-56)
    rng = np.random.default_rng(2)
    wl = scene.Workload("t", 160, 128, seed=11)
    img = np.zeros((128, 160, 4), np.float32)
    img[..., 0] = scene.clean_scene(160, 128, 11)[..., 1] + 0.01 * rng.standard_normal((128, 160))
    b = O.pca_basis(img)
    ev, vec = _numpy_pca_basis(img)
    assert ev[7] > 1.05 * ev[8]  # the 8-D subspace is well separated
    top = vec[:, :8]
    assert np.allclose(top @ (top.T @ b), b, atol=1e-8)
    # unit norm, orthogonal, signed so the largest-magnitude entry is positive
    assert np.allclose(b.T @ b, np.eye(8), atol=1e-10)
    for c in range(8):
        assert b[np.argmax(np.abs(b[:, c])), c] > 0


def test_pca_recovers_rank_k_subspace():
    # interior patches drawn from a rank-3 subspace plus a small isotropic
    # floor: the top-3 eigenvectors span the planted subspace
    rng = np.random.default_rng(3)
    basis, _ = np.linalg.qr(rng.standard_normal((25, 3)))
    h, w = 256, 256
    img = np.zeros((h, w, 4), np.float32)
    for y in range(1, h // 8 - 1):
        for x in range(1, w // 8 - 1):
            patch = (basis @ rng.standard_normal(3)).reshape(5, 5)
            img[8 * y - 2:8 * y + 3, 8 * x - 2:8 * x + 3, 0] = patch
    b = O.pca_basis(img)
    top = b[:, :3]
    assert np.allclose(basis @ (basis.T @ top), top, atol=2e-2)


def test_flat_field_demosaic_is_flat():
    # a constant-colour mosaic demosaics to that colour away from the borders
    wl = scene.Workload("flat", 64, 48, levels=3, gain=1e9, read=0.0, iso=200, seed=1)
    p = scene.make_params(wl)
    clean = np.ones((48, 64, 3), np.float32) * np.array([0.2, 0.3, 0.25], np.float32)
    raw = scene.add_noise(scene.mosaic(clean), wl.black, wl.white, wl.gain, wl.read, 0)
    r = O.raw_pipeline(raw, p, denoise=False, f64=True)
    out = r["out"][8:-8, 8:-8, :3]
    scaled = 0.9 * np.rint(clean[0, 0] * (wl.white - wl.black)) / (wl.white - wl.black) + 0.1
    assert np.allclose(out, scaled, atol=1e-6)


def test_flat_field_denoise_reduces_noise():
    wl = scene.Workload("flat", 128, 96, levels=3, gain=0.8, read=3.0, iso=200, seed=1)
    p = scene.make_params(wl)
    clean = np.full((96, 128, 3), 0.18, np.float32)
    raw = scene.add_noise(scene.mosaic(clean), wl.black, wl.white, wl.gain, wl.read, 5)
    noisy = O.raw_pipeline(raw, p, denoise=False, f64=True)["out"][16:-16, 16:-16, :3]
    den = O.raw_pipeline(raw, p, denoise=True, f64=True)["out"][16:-16, 16:-16, :3]
    assert den.std() < 0.2 * noisy.std()
    assert abs(den.mean() - noisy.mean()) < 2e-3


def test_f32_and_f64_oracles_agree():
    wl = scene.Workload("t", 96, 64, levels=3, gain=0.8, read=3.0, iso=200, seed=3)
    raw, _ = scene.make_raw(wl)
    p = scene.make_params(wl)
    a = O.raw_pipeline(raw, p, f64=True)["out"]
    b = O.raw_pipeline(raw, p, f64=False)["out"]
    assert scene.psnr(a[..., :3], b[..., :3]) > 80
