"""C-ABI checks that need no GPU: the library loads, exports every symbol
include/glscam.h declares, and its host-only functions (calibration,
tap folding) agree with the oracle and the reference's formulas."""
import ctypes as C
import math
import re
from pathlib import Path

import numpy as np
import pytest

import _oracle as O
import glasscamerapublic_b200 as g
from glasscamerapublic_b200 import scene

HEADER = Path(__file__).resolve().parents[1] / "include" / "glscam.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gls_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(native):
    names = declared_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(native, n), n
    assert set(names) == set(g.exported_symbols())


def test_version_string(native):
    assert b"sm_100a" in native.gls_version()


def test_gaussian_taps_match_oracle_bitwise(native):
    for r in (1.5, 4.5, 0.4, 2.0):
        buf = (C.c_float * 300)()
        n = C.c_int32()
        g.check(native.gls_gaussian_bilinear_taps(r, buf, 100, C.byref(n)))
        lib_taps = np.frombuffer(buf, np.float32)[: 3 * n.value].reshape(-1, 3)
        assert np.array_equal(lib_taps, O.gaussian_taps(r))


def test_gaussian_taps_rejects_small_buffer(native):
    buf = (C.c_float * 30)()
    n = C.c_int32()
    assert native.gls_gaussian_bilinear_taps(4.5, buf, 10, C.byref(n)) == g.GLS_ERR_INVALID_ARG
    assert n.value == 25


def _cal(iso):
    return g.iPhone14WideCalibration(levels=5).getDemosaicParameters(iso)


def test_calibration_integer_division_lerp():
    # iPhone14WideCalibration::nlfFromIso uses integer division: inside a
    # bracket the factor is 0, so ISO 150 gives the ISO 100 anchor exactly.
    p100, p150 = _cal(100), _cal(150)
    assert list(p150.raw_nlf.b) == list(p100.raw_nlf.b)
    assert p100.raw_nlf.b[1] == pytest.approx(2.378e-4)
    assert p100.pyramid_nlf[0].b[0] == pytest.approx(3.549e-05)
    # top of the last bracket: (12500 - 6100) / 6100 = 1 -> ISO 12500 anchor
    assert _cal(12500).raw_nlf.b[0] == pytest.approx(1.210e-02)
    assert _cal(20000).raw_nlf.b[0] == pytest.approx(1.210e-02)  # clamped


def test_calibration_denoise_schedule():
    # getDenoiseParameters, iPhone14WideCalibration.cpp:65-119
    for iso in (50, 100, 400, 1600, 12500):
        p = _cal(iso)
        a = min(max((math.log2(iso) - math.log2(50)) / (math.log2(12500) - math.log2(50)), 0), 1)
        lerp = 1 + a
        assert p.denoise[0].luma == pytest.approx(3 * lerp, rel=1e-6)
        assert p.denoise[1].luma == pytest.approx(1.5 * lerp, rel=1e-6)
        assert p.denoise[4].luma == pytest.approx(lerp, rel=1e-6)
        assert p.denoise[0].chroma_boost == 8 and p.denoise[1].chroma_boost == 4 and p.denoise[2].chroma_boost == 2
        ss = min(max((a - 0.3) / 0.3, 0), 1)
        ss = ss * ss * (3 - 2 * ss)
        assert p.denoise[0].gradient_boost == pytest.approx(2 * (2 - ss), rel=1e-6)
        assert p.denoise[0].sharpening == pytest.approx(1.5 + (1.0 - 1.5) * a, rel=1e-6)
        assert p.denoise[2].gradient_boost == 0 and p.denoise[2].gradient_threshold == 1
        assert p.high_noise_image == (1 if iso >= 100 else 0)
        ra = min(max((math.log2(iso) - math.log2(100)) / (math.log2(12500) - math.log2(100)), 0), 1)
        assert p.raw_denoise_strength == pytest.approx(0.5 + 2.5 * ra, rel=1e-6)


def test_calibration_rejects_bad_camera(native):
    p = g.DemosaicParams()
    assert native.gls_calibration_fill(7, 100, C.byref(p)) == g.GLS_ERR_INVALID_ARG
    assert b"camera" in native.gls_last_error_message()
    assert native.gls_calibration_fill(0, 0, C.byref(p)) == g.GLS_ERR_RANGE


def test_workload_params_are_sane():
    wl = scene.WORKLOADS["cfg2_4032x3024"]
    p = scene.make_params(wl)
    assert p.levels == 5 and p.bayer_pattern == g.RGGB
    assert p.scale_mul[0] == pytest.approx(65535.0 / (4095 - 512))
    a, b = scene.raw_nlf(512, 4095, 2.0, 5.0)
    assert p.raw_nlf.b[1] == pytest.approx(b) and p.raw_nlf.a[1] == pytest.approx(a)


def test_scene_is_deterministic():
    wl = scene.Workload("t", 64, 48, seed=5)
    r1, c1 = scene.make_raw(wl)
    r2, c2 = scene.make_raw(wl)
    assert np.array_equal(r1, r2) and np.array_equal(c1, c2)
    assert r1.dtype == np.uint16 and r1.max() <= wl.white
    assert abs(float(c1.mean()) - 0.18) < 0.02
