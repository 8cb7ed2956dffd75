"""A DNG file through the whole path on the GPU: gls_dng_read ->
gls_dng_demosaic_params -> gls_demosaic (noise reduction and display
post-processing), as the reference's pipelineTest demosaicFile and
PyramidFusion runPipeline do (pipelineTest.cpp:110-175,
pyramidFusion.cpp:46-60). The raw comes back bit-exact from the file, and
the output matches the oracle's pipeline on the DNG's parameters to the raw
path's tolerance."""
import sys
from pathlib import Path

import numpy as np
import pytest

import _oracle as O
import glasscamerapublic_b200 as g
from glasscamerapublic_b200 import dng, scene

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))

pytestmark = pytest.mark.gpu


def _dng(tmp_path, w=512, h=384, iso=1600, comp=7, tile=128):
    wl = scene.Workload("dng", w, h, levels=5, gain=0.5, read=3.0, iso=iso, seed=21)
    raw, _ = scene.make_raw(wl)
    info = g.DngInfo()
    info.cfa_pattern[:] = [0, 1, 1, 2]
    info.black_level, info.white_level, info.iso = wl.black, wl.white, iso
    info.has_color_matrix2 = 1
    info.color_matrix2[:] = [0.66, -0.13, -0.07, -0.39, 1.21, 0.17, -0.06, 0.17, 0.55]
    info.has_as_shot_neutral = 1
    info.as_shot_neutral[:] = [0.52, 1.0, 0.61]
    info.make, info.model = b"Apple", b"iPhone 14 Pro"
    f = tmp_path / "frame.dng"
    dng.write_dng(f, raw, info, comp, tile)
    return f, raw


@pytest.mark.parametrize("comp,tile", [(7, 128), (1, 0)])
def test_dng_file_through_the_path(converter, tmp_path, comp, tile):
    f, raw = _dng(tmp_path, comp=comp, tile=tile)
    back, info = dng.read_dng(f)
    assert np.array_equal(back, raw)
    p = dng.demosaic_params(info)
    assert p.bayer_pattern == 2 and p.levels == 5
    out = converter.demosaic(back, p)  # linear camera RGB
    ref = O.raw_pipeline(back, p, denoise=True, f64=False)["out"]
    d = np.abs(out[..., :3].astype(np.float64) - ref[..., :3])
    assert np.quantile(d, 0.999) <= 1e-4, np.quantile(d, 0.999)
    srgb = converter.demosaic(back, p, fp16=True, postProcess=True)
    assert np.isfinite(srgb).all() and srgb[..., :3].min() >= 0 and srgb[..., :3].max() <= 1


def test_burst_of_dng_files_through_the_driver(converter, tmp_path):
    # PyramidFusion's main(): four DNGs found by name, the "_4_" frame the reference
    import torch
    from glasscamerapublic_b200 import burst
    wl = scene.Workload("b", 1024, 768, levels=5, gain=1.5, read=4.0, iso=800, seed=3000)
    raws, cleans, Hs = scene.make_burst(wl, 4)
    raw_dir = tmp_path / "Raw"
    raw_dir.mkdir()
    names = ["IMG_7_4_.dng", "IMG_7_1_.dng", "IMG_7_2_.dng", "IMG_7_3_.dng"]  # frame 0 is the reference
    for raw, name in zip(raws, names):
        info = g.DngInfo()
        info.cfa_pattern[:] = [0, 1, 1, 2]
        info.black_level, info.white_level, info.iso = wl.black, wl.white, wl.iso
        info.has_color_matrix2 = 1
        info.color_matrix2[:] = [0.66, -0.13, -0.07, -0.39, 1.21, 0.17, -0.06, 0.17, 0.55]
        info.make, info.model = b"Apple", b"iPhone 14 Pro"
        dng.write_dng(raw_dir / name, raw, info, 7, 256)
    bursts = burst.find_bursts(burst.parse_directory(raw_dir))
    assert len(bursts) == 1 and [p.rsplit("/", 1)[-1] for p in bursts[0]] == names[1:] + names[:1]
    fused, Hest, out = burst.fuse_burst(converter, bursts[0])
    assert out.endswith("Fusion/IMG_7aRH_fork.tiff")
    errs = [scene.corner_error(He, Ht, wl.width, wl.height) for He, Ht in zip(Hest, Hs[1:])]
    assert max(errs) < 3.0, errs
    got = burst.read_tiff_rgb8(out)
    want = (255 * np.clip(fused.cpu().numpy()[..., :3], 0, 1)).astype(np.uint8)
    assert np.array_equal(got, want)
    p = dng.demosaic_params(dng.read_dng(bursts[0][3])[1])
    ref = converter.demosaic(torch.from_numpy(raws[0].view(np.int16)).cuda(), p, fp16=True, postProcess=True)
    assert scene.psnr(fused.cpu().numpy()[64:-64, 64:-64, :3], ref.float().cpu().numpy()[64:-64, 64:-64, :3]) > 28.0


def test_pipelined_file_conversion_matches_one_at_a_time(converter, tmp_path):
    paths = []
    for k in range(3):
        d = tmp_path / f"{k}"
        d.mkdir()
        f, _ = _dng(d, w=384, h=256)
        paths.append(f)
    got = [(p, o.numpy().copy()) for p, o in dng.convert_files(converter, paths)]
    assert [p for p, _ in got] == [str(p) for p in paths]
    for path, out in got:
        back, info = dng.read_dng(path)
        ref = converter.demosaic(back, dng.demosaic_params(info), fp16=True, out_fp16=True, postProcess=True)
        assert np.array_equal(out, ref)


@pytest.mark.parametrize("half", [False, True])
def test_grayscale_conversion(converter, half):
    import torch
    from glasscamerapublic_b200 import burst
    sys.path.insert(0, str(Path(__file__).resolve().parent))
    from test_burst_driver import _gray_formula
    rng = np.random.default_rng(5)
    rgb = rng.uniform(-0.1, 1.2, (200, 328, 4)).astype(np.float32)
    if half:
        rgb = rgb.astype(np.float16).astype(np.float32)
    t = [1.9, -0.7, -0.2]
    dev = torch.from_numpy(rgb).cuda()
    out = burst.convert_to_grayscale(dev.half() if half else dev, t)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), _gray_formula(rgb, t))
