"""The burst driver of PyramidFusion (PyramidFusion/pyramidFusion.cpp:263-352)
on the library: bursts of four DNG frames found by name, the last frame the
reference; every frame's G and G2 planes (RawChannels) through SURF, each
other frame registered to the reference per channel, the channel
homographies averaged and scaled to full resolution; every frame through
RawConverter::demosaic with noise reduction and display post-processing;
the registered frames averaged into the reference (registerAndFuse with
count i + 1); the result saved as an 8-bit RGB TIFF (saveFusedImage) in
the directory's sibling "Fusion" as <name up to "_4_">aRH_fork.tiff."""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

from . import ImageView, F32, check, lib
from . import dng


def parse_directory(directory) -> list[str]:
    """parseDirectory (pyramidFusion.cpp:36-44): the .dng / .DNG files, sorted."""
    return sorted(str(p) for p in Path(directory).iterdir()
                  if p.is_file() and p.suffix in (".dng", ".DNG"))


def find_bursts(paths) -> list[list[str]]:
    """findBursts (pyramidFusion.cpp:166-195) through gls_find_bursts."""
    n = len(paths)
    arr = (C.c_char_p * max(n, 1))(*[str(p).encode() for p in paths])
    out = np.full(max(n, 1), -1, np.int32)
    nb = C.c_int32(0)
    check(lib().gls_find_bursts(arr, n, out.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(nb)))
    bursts = [[] for _ in range(nb.value)]
    for p, b in zip(paths, out[:n]):
        if b >= 0:
            bursts[b].append(str(p))
    return bursts


def write_tiff_rgb8(path, rgba, stream=None):
    """saveFusedImage: an RGBA float image (numpy or CUDA tensor) as 8-bit RGB TIFF."""
    if isinstance(rgba, np.ndarray):
        a = np.ascontiguousarray(rgba, np.float32)
        v = ImageView(C.c_void_p(a.ctypes.data), a.shape[1], a.shape[0], a.shape[2], F32, a.strides[0])
    else:
        from .api import _ptr, _row_stride
        v = ImageView(C.c_void_p(_ptr(rgba)), rgba.shape[1], rgba.shape[0], rgba.shape[2],
                      F32 if str(rgba.dtype) == "torch.float32" else 1, _row_stride(rgba))
    check(lib().gls_write_tiff_rgb8(str(path).encode(), C.byref(v), None if stream is None else
                                    C.c_void_p(stream.cuda_stream)))


def read_tiff_rgb8(path) -> np.ndarray:
    """The (h, w, 3) uint8 pixels of a TIFF gls_write_tiff_rgb8 wrote."""
    b = Path(path).read_bytes()
    n = int.from_bytes(b[8:10], "little")
    tags = {}
    for i in range(n):
        e = b[10 + 12 * i:22 + 12 * i]
        tag, typ = int.from_bytes(e[0:2], "little"), int.from_bytes(e[2:4], "little")
        val = int.from_bytes(e[8:10], "little") if typ == 3 else int.from_bytes(e[8:12], "little")
        tags[tag] = val
    w, h, off = tags[256], tags[257], tags[273]
    return np.frombuffer(b, np.uint8, w * h * 3, off).reshape(h, w, 3)


def fuse_burst(converter, paths, out_path=None, fp16: bool = True, stream=None):
    """One burst of four DNGs (burst[3] the reference) as PyramidFusion's
    main() fuses it. Returns (fused RGBA float32 CUDA tensor, homographies
    [3][3][3] reference -> frame at full resolution, output path or None)."""
    import torch

    from .registration import SURF, RegisterAndFuseKernel

    if len(paths) != 4:
        raise ValueError("a burst has four frames (pyramidFusion.cpp:286)")
    ref_path = paths[3]
    order = [ref_path] + list(paths[:3])
    frames = [dng.read_dng(p) for p in order]
    raw0, info0 = frames[0]
    params = dng.demosaic_params(info0)  # taken from the reference frame, reused (:46-56)
    h, w = raw0.shape
    dev = torch.device("cuda", torch.cuda.current_device())
    surf = SURF(w // 2, h // 2, max_features=1500, nOctaves=4, nOctaveLayers=2, hessianThreshold=0.02)
    planes = {c: torch.empty((h // 2, w // 2), dtype=torch.float32, device=dev) for c in (1, 3)}
    for f, (raw, info) in enumerate(frames):
        # RawChannels (pyramidFusion.cpp:106-143): exposure 2^BaselineExposure
        surf.raw_channels(raw, info.bayer_pattern, info.black_level, info.white_level,
                          float(2.0 ** info.baseline_exposure), outs=planes, stream=stream)
        surf.detect_slot(planes[1], 2 * f, stream)
        surf.detect_slot(planes[3], 2 * f + 1, stream)
    Hs = surf.register_frames([0, 1], [[2 * f, 2 * f + 1] for f in range(1, 4)], 1.0, 2000, True, stream)
    rgb = [converter.demosaic(torch.from_numpy(raw.view(np.int16)).to(dev), params, fp16=fp16, postProcess=True)
           for raw, _ in frames]
    fused = rgb[0].float().clone()
    fuse = RegisterAndFuseKernel()
    for i in range(3):
        fuse(fused, rgb[i + 1], fused, Hs[i], i + 1, stream=stream)
    torch.cuda.synchronize()
    surf.close()
    if out_path is None:
        out_path = _fused_path(ref_path)
    write_tiff_rgb8(out_path, fused)
    return fused, Hs, str(out_path)


def _fused_path(ref_path) -> Path:
    """saveFusedImage's name: <name up to "_4_">aRH_fork.tiff in the raw
    directory's sibling "Fusion"."""
    stem = Path(ref_path).stem
    base = stem[:stem.find("_4_")] if "_4_" in stem else stem
    out_dir = Path(ref_path).parent.parent / "Fusion"
    out_dir.mkdir(parents=True, exist_ok=True)
    return out_dir / (base + "aRH_fork.tiff")


def fuse_burst_sharded(converter, paths, dist=None, out_path=None, fp16: bool = True, stream=None, device=None):
    """fuse_burst with the burst split over the ranks of a process group
    (one process per GPU): rank 0 reads the reference frame, takes the
    demosaic parameters from its metadata and detects its G and G2
    features, and broadcasts both; member m of [reference, burst[0..2]]
    belongs to rank m % world, which detects, registers, demosaics and
    warps it on its own GPU; the homographies are all-gathered and the
    per-rank running means of the warped frames reduced (sum) to rank 0,
    which writes the TIFF.

    The result is fuse_burst's: the same homographies bit for bit (each
    registration is one member against the same reference features), and
    the mean of the same warped frames summed in another grouping (float
    rounding). As in fuse_burst, the reference frame's own pixels do not
    enter the mean (registerAndFuse with count 1 replaces them). Returns
    (fused RGBA float32 CUDA tensor on rank 0, None elsewhere; homographies
    [3][3][3]; output path on rank 0, None elsewhere). Without a process
    group (or world 1) this is one rank doing every member. device: where
    the frames live (default the current CUDA device)."""
    import torch

    from . import KEYPOINT_DTYPE, DemosaicParams, shard
    from .registration import SURF, RegisterAndFuseKernel, register_image

    if len(paths) != 4:
        raise ValueError("a burst has four frames (pyramidFusion.cpp:286)")
    active = shard._active(dist)
    rank, world = (dist.get_rank(), dist.get_world_size()) if active else (0, 1)
    order = [paths[3]] + list(paths[:3])
    mine = shard.burst_members(len(order), world)[rank]
    frames = {m: dng.read_dng(order[m]) for m in mine}
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    # parameters and image size from the reference frame's metadata
    head = None
    if rank == 0:
        raw0, info0 = frames[0]
        head = bytes(dng.demosaic_params(info0)) + np.array(raw0.shape, np.int64).tobytes()
    head = shard.broadcast_bytes(head, dist)
    psize = C.sizeof(DemosaicParams)
    params = DemosaicParams.from_buffer_copy(head[:psize])
    h, w = (int(v) for v in np.frombuffer(head[psize:], np.int64))
    surf = SURF(w // 2, h // 2, max_features=1500, nOctaves=4, nOctaveLayers=2, hessianThreshold=0.02)
    try:
        planes = {c: torch.empty((h // 2, w // 2), dtype=torch.float32, device=dev) for c in (1, 3)}
        for m in mine:
            raw, info = frames[m]
            if raw.shape != (h, w):
                raise ValueError(f"{order[m]} is {raw.shape[1]}x{raw.shape[0]}, the reference {w}x{h}")
            surf.raw_channels(raw, info.bayer_pattern, info.black_level, info.white_level,
                              float(2.0 ** info.baseline_exposure), outs=planes, stream=stream)
            surf.detect_slot(planes[1], 2 * m, stream)
            surf.detect_slot(planes[3], 2 * m + 1, stream)
        # the reference features: rank 0's slots 0 and 1, broadcast to the others
        for c in (0, 1):
            kf, df = surf.features(c, stream) if rank == 0 else (np.zeros(0, KEYPOINT_DTYPE), np.zeros((0, 64)))
            kb, db = shard.broadcast_features(kf, df, dist)
            if rank != 0:
                if kb.is_cuda:
                    surf.load_features(c, kb, db, stream)
                else:
                    surf.load_features(c, kb.numpy().view(KEYPOINT_DTYPE), db.numpy(), stream)
        members = [m for m in mine if m > 0]
        Hs = (surf.register_frames([0, 1], [[2 * m, 2 * m + 1] for m in members], 1.0, 2000, True, stream)
              if members else np.zeros((0, 3, 3), np.float32))
        Hall = shard.all_gather_rows(Hs.reshape(-1, 9), [m - 1 for m in members], len(order) - 1,
                                     dist).reshape(-1, 3, 3)
        # this rank's running mean of its warped members (registerAndFuse
        # with counts 1, 2, ...; count 1 ignores the fused input)
        part = torch.zeros((h, w, 4), dtype=torch.float32, device=dev)
        fuse = RegisterAndFuseKernel()
        for k, m in enumerate(members):
            raw, _ = frames[m]
            rgb = converter.demosaic(torch.from_numpy(raw.view(np.int16)).to(dev), params, fp16=fp16,
                                     postProcess=True)
            if k == 0:
                register_image(rgb, part, Hall[m - 1], stream=stream)
            else:
                fuse(part, rgb, part, Hall[m - 1], k + 1, stream=stream)
        if dev.type == "cuda":
            torch.cuda.synchronize()
        fused = shard.reduce_mean(part, len(members), len(order) - 1, dist)
    finally:
        surf.close()
    if rank != 0:
        return None, Hall, None
    if out_path is None:
        out_path = _fused_path(paths[3])
    write_tiff_rgb8(out_path, fused)
    return fused, Hall, str(out_path)


def convert_to_grayscale(rgb, transform, out=None, stream=None):
    """convertToGrayscale (demosaic.metal:1707-1723) on a CUDA RGBA tensor:
    max(t . ((rgb - 0.1) / 0.9), 0) as an (h, w) float32 CUDA tensor."""
    import torch

    from .api import _ptr, _row_stride, _stream_handle

    h, w = rgb.shape[:2]
    if out is None:
        out = torch.empty((h, w), dtype=torch.float32, device=rgb.device)
    iv = ImageView(C.c_void_p(_ptr(rgb)), w, h, 4, F32 if rgb.dtype == torch.float32 else 1, _row_stride(rgb))
    ov = ImageView(C.c_void_p(_ptr(out)), w, h, 1, F32, _row_stride(out))
    t = (C.c_float * 3)(*[float(v) for v in transform])
    check(lib().gls_convert_to_grayscale(C.byref(iv), t, C.byref(ov), _stream_handle(stream)))
    return out
