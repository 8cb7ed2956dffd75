"""The burst driver's host side (gls_burst.cpp) on the CPU: findBursts
(pyramidFusion.cpp:166-195) on file names, and saveFusedImage's 8-bit TIFF
(pyramidFusion.cpp:152-164)."""
import numpy as np
import pytest

from glasscamerapublic_b200 import burst


def _find_bursts_reference(paths):
    """findBursts restated: a "_1_" stem opens a burst; later files join when
    their stem shares the prefix up to that position."""
    bursts, cur, first, found = [], [], None, -1
    for p in paths:
        stem = p.rsplit("/", 1)[-1].rsplit(".", 1)[0]
        f = stem.find("_1_")
        if f >= 0:
            first, found = stem, f
            if cur:
                bursts.append(cur)
            cur = [p]
        elif found >= 0 and stem[:found] == first[:found]:
            cur.append(p)
    if cur:
        bursts.append(cur)
    return bursts


def test_find_bursts_groups_by_prefix():
    paths = ["d/x_0.dng",                                     # before any burst: none
             "d/IMG_100_1_a.dng", "d/IMG_100_2_a.dng", "d/IMG_100_3_a.dng", "d/IMG_100_4_a.dng",
             "d/OTHER_2.dng",                                 # another prefix: none
             "d/IMG_200_1_b.dng", "d/IMG_200_2_b.DNG", "d/IMG_200_4_b.dng",
             "d/IMG_300_1_.dng"]
    got = burst.find_bursts(paths)
    assert got == _find_bursts_reference(paths)
    assert got == [paths[1:5], paths[6:9], paths[9:10]]
    assert burst.find_bursts([]) == []
    assert burst.find_bursts(["a.dng", "b.dng"]) == []


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_find_bursts_random_names(seed):
    rng = np.random.default_rng(seed)
    names = []
    for i in range(60):
        pre = rng.choice(["A", "B", "AB", "A_B"])
        mid = rng.choice(["_1_", "_2_", "_3_", "_4_", "_x"])
        names.append(f"dir/{pre}{mid}{i}.dng")
    names.sort()
    assert burst.find_bursts(names) == _find_bursts_reference(names)


def test_tiff_rgb8_is_the_clamped_truncation(tmp_path):
    rng = np.random.default_rng(0)
    img = rng.uniform(-0.2, 1.2, (37, 53, 4)).astype(np.float32)
    f = tmp_path / "f.tiff"
    burst.write_tiff_rgb8(f, img)
    got = burst.read_tiff_rgb8(f)
    want = (255 * np.clip(img[..., :3], 0, 1)).astype(np.uint8)
    assert np.array_equal(got, want)


def _gray_formula(rgb, t):
    """max(t . ((rgb - 0.1) / 0.9), 0) in float32, one rounding per operation."""
    f = np.float32
    p = ((rgb[..., :3].astype(f) - f(0.1)) / f(0.9)).astype(f)
    d = (f(t[0]) * p[..., 0] + f(t[1]) * p[..., 1]).astype(f) + (f(t[2]) * p[..., 2]).astype(f)
    return np.maximum(d.astype(f), f(0))


def test_grayscale_formula_is_the_reference_kernel():
    import _ref as R
    if not R.available():
        pytest.skip("reference kernels not built (make -C oracle ref)")
    import ctypes as C
    L = R.lib()
    fp = C.POINTER(C.c_float)
    L.ref_convert_to_grayscale.argtypes = [fp, C.c_int, C.c_int, fp, fp]
    rng = np.random.default_rng(4)
    rgb = rng.uniform(-0.1, 1.2, (24, 40, 4)).astype(np.float32)
    t = np.array([1.9, -0.7, -0.2], np.float32)
    gray = np.zeros((24, 40), np.float32)
    L.ref_convert_to_grayscale(rgb.ctypes.data_as(fp), 40, 24, t.ctypes.data_as(fp), gray.ctypes.data_as(fp))
    assert np.array_equal(gray, _gray_formula(rgb, t))


def test_burst_drivers_want_four_frames():
    from glasscamerapublic_b200 import burst
    for fn in (burst.fuse_burst, burst.fuse_burst_sharded):
        with pytest.raises(ValueError):
            fn(None, ["a.dng", "b.dng", "c.dng"])
