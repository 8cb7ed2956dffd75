"""DNG ingest (gls_dng.cpp) on the CPU: the library's reader and writer
against an independent restatement of the lossless JPEG codec and the TIFF
layout (oracle/dng_oracle.py, written from the T.81, TIFF 6.0 and DNG 1.4
specifications: the reference's own reader lives in its un-vendored
GlassImage library), and the metadata-to-parameters step against the
reference's unpackDNGMetadata restated (demosaic_utils.cpp:268-366).

Raw samples must round-trip bit for bit; parameters to float rounding.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

import glasscamerapublic_b200 as g
from glasscamerapublic_b200 import dng, scene

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import dng_oracle as D  # noqa: E402

CFA = {0: [1, 0, 2, 1], 1: [1, 2, 0, 1], 2: [0, 1, 1, 2], 3: [2, 1, 1, 0]}  # GRBG, GBRG, RGGB, BGGR
CM2 = [0.7, -0.1, -0.05, -0.3, 1.2, 0.1, -0.05, 0.15, 0.6]


def _raw(w, h, seed=1, bits=12):
    rng = np.random.default_rng(seed)
    base = scene.mosaic(scene.clean_scene(w, h, seed), 2)
    raw = np.clip(base * (2 ** bits - 1) + rng.normal(0, 8, base.shape), 0, 2 ** bits - 1)
    return raw.astype(np.uint16)


def _info(pattern=2, iso=800):
    info = g.DngInfo()
    info.cfa_pattern[:] = CFA[pattern]
    info.black_level, info.white_level, info.iso = 64, 4095, iso
    info.has_color_matrix2 = 1
    info.color_matrix2[:] = CM2
    info.has_as_shot_neutral = 1
    info.as_shot_neutral[:] = [0.5, 1.0, 0.6]
    info.baseline_exposure = 0.5
    info.make, info.model = b"Apple", b"iPhone 14 Pro"
    info.lens_model = b"iPhone 14 Pro back camera 6.86mm f/1.78"
    return info


@pytest.mark.parametrize("comp,tile", [(1, 0), (1, 128), (7, 0), (7, 64), (7, 256)])
@pytest.mark.parametrize("w,h", [(512, 384), (330, 250)])
def test_library_round_trip(tmp_path, comp, tile, w, h):
    raw = _raw(w, h)
    info = _info()
    f = tmp_path / "a.dng"
    dng.write_dng(f, raw, info, comp, tile)
    back, i2 = dng.read_dng(f)
    assert np.array_equal(back, raw)
    assert (i2.width, i2.height, i2.compression, i2.iso, i2.bayer_pattern) == (w, h, comp, 800, 2)
    assert i2.black_level == 64 and i2.white_level == 4095 and i2.baseline_exposure == 0.5
    assert np.allclose(list(i2.color_matrix2), CM2, atol=1e-6) and not i2.has_color_matrix1
    assert np.allclose(list(i2.as_shot_neutral), [0.5, 1.0, 0.6], atol=1e-6)
    assert i2.lens_model == info.lens_model and i2.make == b"Apple"


def test_library_lossless_jpeg_decodes_with_the_independent_decoder(tmp_path):
    # the library's tiles, decoded by the independent decoder
    raw = _raw(64, 48, seed=3, bits=16)
    f = tmp_path / "b.dng"
    dng.write_dng(f, raw, _info(), 7, 32)
    data = f.read_bytes()
    starts = [i for i in range(len(data) - 1) if data[i] == 0xFF and data[i + 1] == 0xD8]
    tiles = []
    for s in starts:
        e = data.index(b"\xff\xd9", s) + 2
        tiles.append(D.lj92_decode(data[s:e]))
    assert len(tiles) == 4  # 2 x 2 tiles of 32 x 32
    got = np.zeros((64, 64), np.uint16)
    for t, tile in enumerate(tiles):
        ty, tx = divmod(t, 2)
        got[32 * ty:32 * ty + 32, 32 * tx:32 * tx + 32] = tile.reshape(32, 32)
    assert np.array_equal(got[:48, :64], raw)


@pytest.mark.parametrize("predictor", [1, 2, 3, 4, 5, 6, 7])
@pytest.mark.parametrize("nc", [1, 2, 4])
def test_reader_decodes_every_predictor_and_interleave(tmp_path, predictor, nc):
    raw = _raw(48, 32, seed=predictor + nc, bits=16)
    f = tmp_path / "c.dng"
    D.write_dng(f, raw, {"cfa": CFA[2], "iso": 200, "cm2": CM2}, compression=7, tile=16, predictor=predictor, nc=nc)
    back, info = dng.read_dng(f)
    assert np.array_equal(back, raw)
    assert info.iso == 200 and info.bayer_pattern == 2


@pytest.mark.parametrize("big_endian", [False, True])
@pytest.mark.parametrize("bps", [16, 12, 14, 10])
def test_reader_layouts(tmp_path, big_endian, bps):
    raw = _raw(40, 24, seed=bps, bits=bps)
    f = tmp_path / "d.dng"
    D.write_dng(f, raw, {"cfa": CFA[3], "iso": 1600, "white": 2 ** bps - 1, "cm1": CM2, "black": 32,
                         "baseline_exposure": -0.25, "neutral": [0.4, 1.0, 0.7]},
                big_endian=big_endian, compression=1, bps=bps, sub_ifd=True)
    back, info = dng.read_dng(f)
    assert np.array_equal(back, raw)
    assert info.bits_per_sample == bps and info.bayer_pattern == 3 and info.white_level == 2 ** bps - 1
    assert info.has_color_matrix1 and not info.has_color_matrix2 and info.black_level == 32
    assert info.baseline_exposure == pytest.approx(-0.25)


def test_reader_finds_the_raw_image_behind_a_thumbnail_in_lossless_strips(tmp_path):
    raw = _raw(64, 40, seed=9, bits=14)
    f = tmp_path / "e.dng"
    D.write_dng(f, raw, {"cfa": CFA[0], "iso": 400, "cm2": CM2}, big_endian=True, compression=7, tile=0,
                predictor=6, nc=2, sub_ifd=True)
    back, info = dng.read_dng(f)
    assert np.array_equal(back, raw) and info.bayer_pattern == 0


@pytest.mark.parametrize("neutral", [True, False])
@pytest.mark.parametrize("be", [0.0, 0.5, -1.0])
def test_parameters_follow_unpack_dng_metadata(tmp_path, neutral, be):
    info = _info(pattern=0, iso=800)
    info.has_as_shot_neutral = int(neutral)
    info.baseline_exposure = be
    p = dng.demosaic_params(info)
    bayer, em, rgb_cam, scale = D.unpack_dng_metadata(CM2, [0.5, 1.0, 0.6] if neutral else None, 64, 4095, be,
                                                      CFA[0], list(p.xyz_rgb))
    assert p.bayer_pattern == bayer == 0
    assert p.exposure_multiplier == pytest.approx(em)
    assert np.allclose(np.array(p.rgb_cam).reshape(3, 3), rgb_cam, rtol=2e-6, atol=2e-6)
    assert np.allclose(list(p.scale_mul), scale, rtol=1e-6)
    assert p.black_level == 64 and p.white_level == 4095
    # and the camera's calibration at the DNG's ISO
    ref = scene.make_params(scene.Workload("x", 64, 64, iso=800))
    g.check(g.lib().gls_calibration_fill(g.CAMERA_IPHONE14_WIDE, 800, __import__("ctypes").byref(ref)))
    assert list(p.raw_nlf.a) == list(ref.raw_nlf.a) and p.denoise[0].luma == ref.denoise[0].luma


def test_camera_selection():
    info = _info()
    assert dng.camera(info) == g.CAMERA_IPHONE14_WIDE
    info.model = b"Pixel 7"
    assert dng.camera(info) == -1


def test_bad_files_are_status_codes(tmp_path):
    f = tmp_path / "x.dng"
    f.write_bytes(b"not a tiff at all")
    with pytest.raises(g.GlsError) as e:
        dng.read_dng(f)
    assert e.value.code == g.GLS_ERR_INVALID_ARG
    with pytest.raises(g.GlsError):
        dng.read_dng(tmp_path / "missing.dng")
    # a valid TIFF without a CFA image
    raw = _raw(16, 16)
    D.write_dng(f, raw, {"cfa": CFA[2]}, compression=1)
    data = bytearray(f.read_bytes())
    i = data.find((32803).to_bytes(2, "little"))
    data[i:i + 2] = (2).to_bytes(2, "little")  # photometric RGB
    f.write_bytes(bytes(data))
    with pytest.raises(g.GlsError) as e:
        dng.read_dng(f)
    assert e.value.code == g.GLS_ERR_UNSUPPORTED
    # a truncated lossless JPEG tile
    D.write_dng(f, raw, {"cfa": CFA[2]}, compression=7, tile=16)
    data = f.read_bytes()
    cut = data.index(b"\xff\xda") + 20
    f.write_bytes(data[:cut] + b"\xff\xd9" + data[cut + 2:])
    try:
        back, _ = dng.read_dng(f)
        assert not np.array_equal(back, raw)
    except g.GlsError:
        pass
