"""A burst split over ranks (burst.fuse_burst_sharded) against the one-rank
burst driver (burst.fuse_burst) on the same four DNG files.

  * gls_surf_load_features: features loaded into a slot (from host or
    device memory) match like the detected ones, bit for bit;
  * one rank: the split driver is fuse_burst, bit for bit;
  * two gloo ranks, both on this GPU: the homographies are fuse_burst's bit
    for bit, the fused frame its mean summed in another grouping (max
    |diff| <= 2e-6 on [0, 1] values).

The two ranks share one GPU: their kernels never wait on one another (the
collectives run on the host, over gloo), so they may interleave in any
order. The NCCL path moves the same tensors on the GPU instead; it is not
exercised here, where a run holds one GPU.
"""
import os
import socket

import numpy as np
import pytest

import glasscamerapublic_b200 as g
from glasscamerapublic_b200 import dng, scene

pytestmark = pytest.mark.gpu

CM2 = [0.66, -0.13, -0.07, -0.39, 1.21, 0.17, -0.06, 0.17, 0.55]


def _burst_files(tmp_path, w=1024, h=768):
    wl = scene.Workload("b", w, h, levels=5, gain=1.5, read=4.0, iso=800, seed=3100)
    raws, _, Hs = scene.make_burst(wl, 4)
    raw_dir = tmp_path / "Raw"
    raw_dir.mkdir()
    names = ["IMG_9_4_.dng", "IMG_9_1_.dng", "IMG_9_2_.dng", "IMG_9_3_.dng"]  # frame 0 is the reference
    for raw, name in zip(raws, names):
        info = g.DngInfo()
        info.cfa_pattern[:] = [0, 1, 1, 2]
        info.black_level, info.white_level, info.iso = wl.black, wl.white, wl.iso
        info.has_color_matrix2 = 1
        info.color_matrix2[:] = CM2
        info.make, info.model = b"Apple", b"iPhone 14 Pro"
        dng.write_dng(raw_dir / name, raw, info, 7, 256)
    from glasscamerapublic_b200 import burst
    return burst.find_bursts(burst.parse_directory(raw_dir))[0], Hs


def test_loaded_features_match_like_detected():
    import torch
    from glasscamerapublic_b200 import KEYPOINT_DTYPE, scene as S
    from glasscamerapublic_b200.registration import SURF
    wl = S.Workload("f", 512, 384, levels=5, gain=1.5, read=4.0, iso=800, seed=3200)
    raws, _, _ = S.make_burst(wl, 2)
    surf = SURF(256, 192, max_features=1500)
    try:
        planes = {c: torch.empty((192, 256), dtype=torch.float32, device="cuda") for c in (1, 3)}
        for f in range(2):
            surf.raw_channels(raws[f], 2, wl.black, wl.white, 1.0, outs=planes)
            surf.detect_slot(planes[1], 2 * f)
        kps, desc = surf.features(0)
        assert len(kps) > 50
        surf.load_features(9, kps, desc)  # host memory
        kb = torch.from_numpy(kps.view(np.uint8).copy()).cuda()
        surf.load_features(10, kb, torch.from_numpy(desc).cuda())  # device memory
        torch.cuda.synchronize()
        want = surf.match_slots(0, 2)
        for slot in (9, 10):
            k2, d2 = surf.features(slot)
            assert k2.tobytes() == kps.tobytes() and np.array_equal(d2, desc)
            assert surf.match_slots(slot, 2).tobytes() == want.tobytes()
        with pytest.raises(g.GlsError):
            surf.load_features(11, np.zeros(1501, KEYPOINT_DTYPE), np.zeros((1501, 64), np.float32))
        with pytest.raises(g.GlsError):
            surf.load_features(32, kps, desc)
    finally:
        surf.close()


def test_one_rank_is_the_burst_driver(converter, tmp_path):
    from glasscamerapublic_b200 import burst
    paths, _ = _burst_files(tmp_path)
    fused, Hs, _ = burst.fuse_burst(converter, paths, out_path=tmp_path / "a.tiff")
    fused2, Hs2, out2 = burst.fuse_burst_sharded(converter, paths, out_path=tmp_path / "b.tiff")
    assert np.array_equal(Hs, Hs2)
    assert np.array_equal(fused.cpu().numpy(), fused2.cpu().numpy())
    assert burst.read_tiff_rgb8(tmp_path / "a.tiff").tobytes() == burst.read_tiff_rgb8(out2).tobytes()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, paths, out_dir, q):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        from glasscamerapublic_b200 import burst
        conv = g.RawConverter(0)
        try:
            fused, Hs, out = burst.fuse_burst_sharded(conv, paths, dist, out_path=os.path.join(out_dir, "s.tiff"))
        finally:
            conv.close()
        if rank == 0:
            np.save(os.path.join(out_dir, "fused.npy"), fused.cpu().numpy())
        q.put((rank, Hs.tolist(), fused is None, out))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_the_burst(converter, tmp_path):
    import torch.multiprocessing as mp
    from glasscamerapublic_b200 import burst
    paths, Htrue = _burst_files(tmp_path)
    fused, Hs, _ = burst.fuse_burst(converter, paths, out_path=tmp_path / "a.tiff")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, paths, str(tmp_path), q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank, H, none, out in res:
        assert np.array_equal(np.asarray(H, np.float32), Hs), rank  # every rank has every homography
        assert none == (rank != 0) and (out is None) == (rank != 0)
    got = np.load(tmp_path / "fused.npy")
    want = fused.cpu().numpy()
    assert np.abs(got - want).max() <= 2e-6, np.abs(got - want).max()
    errs = [scene.corner_error(He, Ht, 1024, 768) for He, Ht in zip(Hs, Htrue[1:])]
    assert max(errs) < 3.0, errs
