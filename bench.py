#!/usr/bin/env python3
"""Benchmark of the raw -> RGB hot path (demosaic + 5-level PCA pyramid
denoise + reconstruct) on 12 MP RGGB frames.

A step is one batch of six frames of the 4032x3024 12-bit workload through
the batched RawConverter::demosaic with noise reduction, on the FP16-storage
path (frames run concurrently on three streams). `value` is frames/s with
the raw frames already resident in HBM; `e2e` is the same batched call with
host buffers (pinned raw in, FP16 RGBA out) copied inside the timed region. With --gpus N (torchrun), every rank converts its own
frames (no data-path collective); the time is the max over ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "12MP raw->RGB frames/s (demosaic + 5-level PCA pyramid denoise), FP16-storage batched path"
UNIT = "frames/s"
WORKLOAD = "cfg2_4032x3024"
N_ROTATE = 6  # distinct resident frames (6 x 24 MB raw + planes >> 126 MB L2)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-full-frame", action="store_true", help="reference arm: skip the one whole-frame check")
    ap.add_argument("--workload", default=WORKLOAD, help="workload name (cfg2_4032x3024 or cfg1_1024x768)")
    ap.add_argument("--quick", action="store_true", help="timed FP16 loop only (for profiler captures)")
    ap.add_argument("--frames", type=int, default=N_ROTATE, help="frames per step (batch size)")
    ap.add_argument("--no-burst", action="store_true", help="skip the burst registration + fusion leg")
    ap.add_argument("--burst-frames", type=int, default=8)
    ap.add_argument("--burst-only", action="store_true", help="run only the burst leg (for profiler captures)")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint (calibration-gradient) leg")
    ap.add_argument("--adjoint-only", action="store_true", help="run only the adjoint leg (for profiler captures)")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-sensor batch leg")
    ap.add_argument("--mixed-only", action="store_true", help="run only the mixed-sensor batch leg")
    ap.add_argument("--no-post", action="store_true", help="skip the display post-processing leg")
    ap.add_argument("--post-only", action="store_true", help="run only the post-processing leg")
    ap.add_argument("--post-frames", type=int, default=N_ROTATE, help="frames per batch of the post-processing leg")
    ap.add_argument("--no-dng", action="store_true", help="skip the DNG-file leg")
    ap.add_argument("--dng-only", action="store_true", help="run only the DNG-file leg")
    ap.add_argument("--no-calibrate", action="store_true", help="skip the noise-model measurement leg")
    ap.add_argument("--calibrate-only", action="store_true", help="run only the noise-model measurement leg")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for k, n in enumerate(names):
                    if r[5 + k].lower().startswith("active"):
                        reasons.add(n)
            except (ValueError, IndexError):
                pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


TILES = 4  # the CPU baseline's sample: one of the 4 x 4 full-resolution tiles of a frame


def cpu_frame_setup(wl):
    """The reference's path on the host cores, set up on one full frame of
    the workload: (run_tile(i), kind, what, threads, tile size). run_tile(i)
    converts tile i of the frame's TILES x TILES full-resolution tiles
    (1008x756 of 4032x3024) with the same scene, noise, ISO and 5-level
    schedule, so TILES^2 tiles are the frame's pixel work. It runs the
    reference's own Metal kernels compiled for the CPU with the parameters
    of the reference's own iPhone14WideCalibration (oracle/_ref, kind
    "reference") where they were built, else the oracle's FP32 restatement
    (kind "port"). Nothing of the library under test is loaded on the
    reference path."""
    sys.path.insert(0, str(ROOT / "tests"))
    import _oracle as O
    import _ref as R
    from glasscamerapublic_b200 import scene
    raw, _ = scene.make_raw(wl)
    threads = os.cpu_count() or 1
    tw, th = wl.width // TILES, wl.height // TILES
    tiles = [np.ascontiguousarray(raw[j * th:(j + 1) * th, i * tw:(i + 1) * tw])
             for j in range(TILES) for i in range(TILES)]
    if R.available():
        kind, what = "reference", "reference Metal kernels and iPhone14WideCalibration compiled for the CPU"
        p = scene.make_params(wl, calibration=R.iPhone14WideCalibration(levels=wl.levels))
        R.lib().ref_set_threads(threads)
        run_tile = lambda i: R.raw_pipeline(tiles[i % len(tiles)], p, denoise=True)
        run_frame = lambda: R.raw_pipeline(raw, p, denoise=True)
    else:
        kind, what = "port", "FP32 oracle"
        p = scene.make_params(wl)
        O.lib().orc_set_threads(threads)
        run_tile = lambda i: O.raw_pipeline(tiles[i % len(tiles)], p, denoise=True, f64=False)
        run_frame = lambda: O.raw_pipeline(raw, p, denoise=True, f64=False)
    return run_tile, run_frame, kind, what, threads, (tw, th)


def cpu_baseline(wl, seconds: float):
    """The reference's path on all host cores over a bounded sample of the
    workload: consecutive full-resolution tiles of one 12 MP frame
    (cpu_frame_setup) for about `seconds`; frames/s = tiles/s / TILES^2."""
    run_tile, _, kind, what, threads, (tw, th) = cpu_frame_setup(wl)
    run_tile(0)  # first-touch of the harness's buffers, untimed
    t0 = time.perf_counter()
    n = 0
    while True:
        run_tile(n)
        n += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    return {"value": n / dt / (TILES * TILES), "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"{n} consecutive {tw}x{th} full-resolution tiles (1/{TILES * TILES} each) of a "
                      f"{wl.width}x{wl.height} frame, 5 levels, {what}, {dt:.1f}s; frames/s = tiles/s / "
                      f"{TILES * TILES}",
            "registration": cpu_registration_baseline(threads)}


def fp64_check_leg(wl, raw, clean, out16, out32):
    """The error of one frame's outputs against the FP64 oracle (the
    checker, run on the host cores outside every timed region): PSNR
    against the FP64 output, the PSNR delta against the clean scene
    (PSNR(out, clean) - PSNR(FP64, clean)) and the max |diff|, for the
    FP16-storage batched path (what `value` times) and the FP32 plain path."""
    sys.path.insert(0, str(ROOT / "tests"))
    import _oracle as O
    from glasscamerapublic_b200 import scene
    O.lib().orc_set_threads(os.cpu_count() or 1)
    p = scene.make_params(wl)
    t0 = time.perf_counter()
    ref = O.raw_pipeline(raw, p, denoise=True, f64=True)["out"][..., :3].astype(np.float64)
    dt = time.perf_counter() - t0
    tgt = scene.target_rgb(clean)
    ps_ref = scene.psnr(ref, tgt)

    def err(out):
        o = np.asarray(out[..., :3], np.float64)
        return {"psnr_db": scene.psnr(o, ref), "delta_psnr_db": scene.psnr(o, tgt) - ps_ref,
                "max_abs": float(np.abs(o - ref).max()), "psnr_vs_clean_db": scene.psnr(o, tgt)}

    return {"fp16_batched": err(out16), "fp32_plain": err(out32), "fp64_psnr_vs_clean_db": ps_ref,
            "gate_delta_psnr_db": 0.05, "frame": f"{wl.width}x{wl.height}, {wl.levels} levels, ISO {wl.iso}",
            "oracle_seconds": dt}


def cpu_registration_baseline(threads: int):
    """The burst workload's registration of one frame on the host cores:
    SURF detect + describe on its G and G2 planes (2016x1512, 1500
    features), matching against the reference frame's features, and
    FindHomography (2000 RANSAC iterations + least squares) per channel,
    as pyramidFusion.cpp:318-346 does per frame. It runs the reference's own
    registration code compiled for the CPU (oracle/_ref/libglsref_reg.so,
    kind "reference") where it was built, else the oracle (kind "port").
    RawChannels is done before the clock starts."""
    sys.path.insert(0, str(ROOT / "tests"))
    import _oracle as O
    import _oracle_reg as OR
    import _ref_reg as F
    from glasscamerapublic_b200 import scene
    wl = scene.WORKLOADS["cfg3_burst_4032x3024"]
    raws, _, _ = scene.make_burst(wl, 2)
    planes = [[OR.raw_channel(r, wl.pattern, c, float(wl.black), float(wl.white)) for c in (1, 3)] for r in raws]
    if F.available():
        kind, what = "reference", "reference SURF.metal / SURF.cpp / Homography.cpp compiled for the CPU"
        F.lib().ref_reg_set_threads(threads)
        det, mat = F.detect, F.match
        fh = lambda p1, p2: F.find_homography(p1, p2, 1.0, 2000)
    else:
        kind, what = "port", "registration oracle"
        O.lib().orc_set_threads(threads)
        det, mat = OR.detect, OR.match
        fh = lambda p1, p2: OR.find_homography(p1, p2, 1.0, 2000)[:2]
    ref = [det(pl) for pl in planes[0]]
    t0 = time.perf_counter()
    for c in range(2):
        k2, d2, _ = det(planes[1][c])
        k1, d1, _ = ref[c]
        m = mat(d1, d2)
        p1 = np.stack([k1["x"][m["query_idx"]], k1["y"][m["query_idx"]]], 1)
        p2 = np.stack([k2["x"][m["train_idx"]], k2["y"][m["train_idx"]]], 1)
        fh(p1, p2)
    ms = 1e3 * (time.perf_counter() - t0)
    return {"ms_per_frame": ms, "cores": threads, "kind": kind,
            "sample": f"one burst frame: 2 x (detect 2016x1512 + match + RANSAC 2000), {what}"}


def burst_leg(args, rank, local, conv, stream):
    """Burst registration and fusion (the 8-frame 4032x3024 burst workload),
    as PyramidFusion/pyramidFusion.cpp:276-346 drives it: every frame through
    the batched raw -> RGB path; RawChannels G and G2 at half resolution;
    SURF detect + describe on each, matched against the reference frame's,
    RANSAC + least-squares homography per channel, averaged, scaled to full
    resolution; then registerAndFuse into an FP32 running mean (count i + 1,
    so the reference frame stays in the mean). Returns device-timed ms per
    burst, the per-stage split and the homography corner errors against the
    known warps."""
    import torch

    from glasscamerapublic_b200 import scene
    from glasscamerapublic_b200.registration import SURF, RegisterAndFuseKernel, fuse_pyramid

    wl = scene.WORKLOADS["cfg3_burst_4032x3024"]
    n = args.burst_frames
    bwl = scene.Workload(wl.name, wl.width, wl.height, levels=wl.levels, black=wl.black, white=wl.white,
                         gain=wl.gain, read=wl.read, iso=wl.iso, pattern=wl.pattern, seed=wl.seed + 97 * rank,
                         extra=wl.extra)
    raws_host, cleans, Hs = scene.make_burst(bwl, n)
    params = scene.make_params(bwl)
    W, H = bwl.width, bwl.height
    dev = f"cuda:{local}"
    raws = [torch.from_numpy(r.view(np.int16)).to(dev) for r in raws_host]
    outs = [torch.empty((H, W, 4), dtype=torch.float16, device=dev) for _ in range(n)]
    fused = torch.empty((H, W, 4), dtype=torch.float32, device=dev)
    surf = SURF(W // 2, H // 2, max_features=1500)
    planes = {c: torch.empty((H // 2, W // 2), dtype=torch.float32, device=dev) for c in (1, 3)}
    fuse = RegisterAndFuseKernel()
    est = [np.eye(3, dtype=np.float32)]
    ev = {k: torch.cuda.Event(enable_timing=True) for k in ("a", "b", "c", "d")}
    black, white = float(bwl.black), float(bwl.white)

    def step():
        ev["a"].record(stream)
        conv.demosaic_batch(raws, [params] * n, outs, fp16=True, out_fp16=True, stream=stream)
        ev["b"].record(stream)
        # G and G2 planes of every frame into feature slots 2f, 2f + 1
        for f in range(n):
            surf.raw_channels(raws[f], bwl.pattern, black, white, 1.0, outs=planes, stream=stream)
            surf.detect_slot(planes[1], 2 * f, stream)
            surf.detect_slot(planes[3], 2 * f + 1, stream)
        fused.copy_(outs[0].float())
        Hfull = surf.register_frames([0, 1], [[2 * f, 2 * f + 1] for f in range(1, n)], 1.0, 2000, True, stream)
        ev["c"].record(stream)
        for i in range(1, n):
            fuse(fused, outs[i], fused, Hfull[i - 1], i + 1, stream=stream)
        ev["d"].record(stream)
        return Hfull

    with torch.cuda.stream(stream):
        for _ in range(max(1, min(args.warmup, 2))):
            Hfull = step()
        stream.synchronize()
        reps = max(2, min(args.steps, 5))
        tot = {"raw_to_rgb": 0.0, "registration": 0.0, "fusion": 0.0, "wall": 0.0}
        for _ in range(reps):
            t0 = time.perf_counter()
            Hfull = step()
            stream.synchronize()
            tot["wall"] += 1e3 * (time.perf_counter() - t0)
            tot["raw_to_rgb"] += ev["a"].elapsed_time(ev["b"])
            tot["registration"] += ev["b"].elapsed_time(ev["c"])
            tot["fusion"] += ev["c"].elapsed_time(ev["d"])
    # pyramid fusion of the same registered burst (uniform and robust weights)
    pfused = torch.empty((H, W, 4), dtype=torch.float32, device=dev)
    Hlist = [np.eye(3, dtype=np.float32)] + list(Hfull)
    pf = {}
    with torch.cuda.stream(stream):
        for rob in (0.0, 100.0):
            fuse_pyramid(surf, outs, Hlist, pfused, levels=5, robustness=rob, stream=stream)
            stream.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fuse_pyramid(surf, outs, Hlist, pfused, levels=5, robustness=rob, stream=stream)
            e1.record(stream)
            stream.synchronize()
            pf[rob] = (e0.elapsed_time(e1), pfused.cpu().numpy()[..., :3])
    errs = [scene.corner_error(Hf, Ht, W, H) for Hf, Ht in zip(Hfull, Hs[1:])]
    # the same registration with the corrected detector (untimed), for its accuracy
    surf.corrected = True
    with torch.cuda.stream(stream):
        for f in range(n):
            surf.raw_channels(raws[f], bwl.pattern, black, white, 1.0, outs=planes, stream=stream)
            surf.detect_slot(planes[1], 2 * f, stream)
            surf.detect_slot(planes[3], 2 * f + 1, stream)
        Hcorr = surf.register_frames([0, 1], [[2 * f, 2 * f + 1] for f in range(1, n)], 1.0, 2000, True, stream)
    surf.corrected = False
    errs_corr = [scene.corner_error(Hf, Ht, W, H) for Hf, Ht in zip(Hcorr, Hs[1:])]
    target = scene.target_rgb(cleans[0])
    fused_np = fused.cpu().numpy()[..., :3]
    single = outs[0].float().cpu().numpy()[..., :3]
    m = 64  # ignore the border, where warped frames clamp
    crop = (slice(m, H - m), slice(m, W - m))
    res = {k: v / reps for k, v in tot.items()}
    surf.close()
    return {
        "workload": f"{n} x {W}x{H} RGGB 12-bit burst (rotation <= 1 deg, shift <= 20 px, perspective <= 1e-5)",
        "ms_per_burst": res["wall"],
        "ms": {"raw_to_rgb": res["raw_to_rgb"], "registration": res["registration"], "fusion": res["fusion"]},
        "registration_ms_per_frame": res["registration"] / (n - 1),
        "corner_error_px": {"max": max(errs), "mean": float(np.mean(errs))},
        "corner_error_px_corrected_detector": {"max": max(errs_corr), "mean": float(np.mean(errs_corr))},
        "fused_psnr_db": scene.psnr(fused_np[crop], target[crop]),
        "pyramid_fusion": {"ms_uniform": pf[0.0][0], "ms_robust": pf[100.0][0], "levels": 5,
                           "psnr_uniform_db": scene.psnr(pf[0.0][1][crop], target[crop]),
                           "psnr_robust_db": scene.psnr(pf[100.0][1][crop], target[crop])},
        "single_frame_psnr_db": scene.psnr(single[crop], target[crop]),
        "note": "SURF on G and G2 at 2016x1512, 1500 features, the reference's detector; all frames x channels "
                "matched and RANSAC'd (2000 iterations, FP64 least squares) in one batch on the GPU; one host "
                "sync per burst",
    }


def adjoint_leg(args, rank, local, conv, stream):
    """Differentiable calibration (the 8 x 2048x1536 adjoint workload): per
    frame, the FP32 raw -> RGB forward and the hand-written adjoint
    (gls_demosaic_denoise_vjp), MSE against the known clean target, gradient
    for the 32 parameters. A step is one pass over the rank's 8 frames and
    ends with the data-parallel exchange: the all-reduce of the ranks'
    gradient sums into the mean gradient (shard.mean_gradient). Device-timed;
    the forward alone is timed too, so the adjoint's own cost is the
    difference."""
    import torch
    import torch.distributed as dist

    from glasscamerapublic_b200 import scene
    from glasscamerapublic_b200 import adjoint as A
    from glasscamerapublic_b200.shard import mean_gradient

    n = 8
    wl = scene.Workload("cfg5_2048x1536", 2048, 1536, levels=5, gain=1.0, read=4.0, iso=800, seed=5000 + 97 * rank)
    params = scene.make_params(wl)
    dev = f"cuda:{local}"
    raws, targets = [], []
    for f in range(n):
        raw, clean = scene.make_raw(wl, frame=f)
        raws.append(torch.from_numpy(raw.view(np.int16)).to(dev))
        targets.append(torch.from_numpy(scene.target_rgb(clean).astype(np.float32)).to(dev))
    out = torch.empty((wl.height, wl.width, 4), dtype=torch.float32, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    import glasscamerapublic_b200 as g
    torch.cuda.synchronize()
    # a converter of its own, so that its buffers are the adjoint's alone
    conv = g.RawConverter(local)
    lib0, _ = g.device_memory(reset_peak=True)
    torch.cuda.reset_peak_memory_stats(dev)
    with torch.cuda.stream(stream):
        for f in range(2):
            A.loss_and_grad(conv, raws[f], params, targets[f], stream=stream)
        reps = max(1, min(args.steps, 3))
        t0 = time.perf_counter()
        e0.record(stream)
        gsum = np.zeros(32)
        lsum = 0.0
        for _ in range(reps):
            step = np.zeros(32)
            for f in range(n):
                loss, grad = A.loss_and_grad(conv, raws[f], params, targets[f], stream=stream)
                step += grad
                lsum += loss
            gsum += mean_gradient(step, n, dist)
        e1.record(stream)
        stream.synchronize()
        wall = (time.perf_counter() - t0) / reps
        ms_vjp = max(e0.elapsed_time(e1) / reps, 1e3 * wall)
        _, lib_peak = g.device_memory()
        lib_peak -= lib0  # the other converters' buffers, held throughout
        torch_peak = torch.cuda.max_memory_allocated(dev)
        e0.record(stream)
        for _ in range(reps):
            for f in range(n):
                conv.demosaic(raws[f], params, noiseReduction=True, fp16=False, out=out, out_fp16=False,
                              stream=stream, sync=False)
        e1.record(stream)
        stream.synchronize()
        ms_fwd = e0.elapsed_time(e1) / reps
    conv.close()
    return {
        "workload": f"{n} x 2048x1536 RGGB 12-bit, 5 levels, FP32 forward + adjoint, MSE vs clean target",
        "ms_per_batch": ms_vjp,
        "ms_per_frame": ms_vjp / n,
        "forward_ms_per_frame": ms_fwd / n,
        "adjoint_ms_per_frame": (ms_vjp - ms_fwd) / n,
        "params_differentiated": 32,
        "device_memory_gb": {"library_peak": lib_peak / 1e9, "torch_peak": torch_peak / 1e9,
                             "total_peak": (lib_peak + torch_peak) / 1e9, "limit": 8.0,
                             "note": "peak over the 8-frame batch's forward + adjoint: the buffers of the leg's own "
                                     "converter (gls_device_memory, over what the process held before) plus "
                                     "torch's (inputs, targets); frames are differentiated one at a time, so the "
                                     "batch holds one frame's activations"},
        "mean_loss": lsum / (reps * n),
        "grad_norm": float(np.linalg.norm(gsum / reps)),
        "ranks_in_gradient": dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1,
        "note": "per-level luma/chroma strengths and YCbCr NLF (A_Y, B_Y, A_C, B_C) by the reverse sweep; "
                "raw-green NLF (a, b) by forward-mode tangents through the front end dotted with dL/d(despeckled "
                "image); PCA bases held fixed",
    }


def mixed_leg(args, rank, local, conv, stream):
    """The 16-frame mixed-sensor batch (4 x 4032x3024, 4 x 6000x4000,
    4 x 5472x3648, 4 x 8368x5584; 12- and 14-bit; per-frame noise model)
    through gls_demosaic_batch on the FP16 path with demosaic + 5-level
    denoise, recorded once as a CUDA graph and replayed. Frames are made on
    the GPU from one seeded scene, resampled to each size, mosaicked, with
    Poisson-Gaussian noise of the frame's sensor."""
    import torch
    import torch.nn.functional as F

    from glasscamerapublic_b200 import block_match_tiles, scene

    dev = f"cuda:{local}"
    wls = scene.mixed_batch(4)
    gen = torch.Generator(device=dev)
    gen.manual_seed(4000 + rank)
    base = torch.from_numpy(scene.clean_scene(2048, 1536, 4000 + rank)).to(dev).permute(2, 0, 1)[None]
    raws, params, outs = [], [], []
    for wl in wls:
        img = F.interpolate(base, size=(wl.height, wl.width), mode="bilinear", align_corners=False)[0]
        m = torch.empty((wl.height, wl.width), device=dev)
        chan = (0, 1, 2, 1)
        for c, (ox, oy) in enumerate(scene.BAYER_OFFSETS[wl.pattern]):
            m[oy::2, ox::2] = img[chan[c], oy::2, ox::2]
        dn = m.clamp(0, 1) * (wl.white - wl.black)
        e = torch.poisson(dn * wl.gain, generator=gen)
        noisy = e / wl.gain + torch.randn(m.shape, device=dev, generator=gen) * wl.read + wl.black
        raw = noisy.round().clamp(0, wl.white).to(torch.int32).to(torch.int16)
        raws.append(raw.contiguous())
        params.append(scene.make_params(wl))
        outs.append(torch.empty((wl.height, wl.width, 4), dtype=torch.float16, device=dev))
        del img, m, dn, e, noisy
    mpix = sum(wl.width * wl.height for wl in wls) / 1e6
    import glasscamerapublic_b200 as g
    import ctypes as C

    def launches():
        st = (g.KernelStat * 32)()
        n = C.c_int32()
        g.check(g.lib().gls_converter_stats(conv.handle, st, 32, C.byref(n)))
        return sum(int(st[i].launches) for i in range(n.value))

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        conv.demosaic_batch(raws, params, outs, stream=stream)  # sizes the slot planes
        stream.synchronize()
        l0 = launches()
        conv.demosaic_batch(raws, params, outs, stream=stream, graph=True)  # runs and records
        stream.synchronize()
        per_batch = (launches() - l0) // 2  # the run and the recording each count once
        for _ in range(2):
            conv.demosaic_batch(raws, params, outs, stream=stream, graph=True)
        stream.synchronize()
        reps = max(2, min(args.steps, 5))
        e0.record(stream)
        for _ in range(reps):
            conv.demosaic_batch(raws, params, outs, stream=stream, graph=True)
        e1.record(stream)
        stream.synchronize()
        ms_graph = e0.elapsed_time(e1) / reps
        e0.record(stream)
        for _ in range(reps):
            conv.demosaic_batch(raws, params, outs, stream=stream)
        e1.record(stream)
        stream.synchronize()
        ms_stream = e0.elapsed_time(e1) / reps
        # the persistent batch: the front ends on the slot streams, then one
        # launch for every pyramid level of every frame, recorded as a graph
        conv.demosaic_batch(raws, params, outs, stream=stream, persistent=True)  # builds the work list
        stream.synchronize()
        l0 = launches()
        conv.demosaic_batch(raws, params, outs, stream=stream, persistent=True)
        per_batch_persistent = launches() - l0
        conv.demosaic_batch(raws, params, outs, stream=stream, persistent=True, graph=True)  # runs and records
        ms_p = []
        for _ in range(reps):
            e0.record(stream)
            conv.demosaic_batch(raws, params, outs, stream=stream, persistent=True, graph=True)  # replays
            e1.record(stream)
            stream.synchronize()
            ms_p.append(e0.elapsed_time(e1))
        ms_persistent = float(np.median(ms_p))
        # strong scaling: the one 16-frame batch split over the ranks by
        # pixel count (shard.assign_frames); this rank's share as its own graph
        from glasscamerapublic_b200.shard import assign_frames
        world = dist_env()[1]
        mine = assign_frames([(wl.width, wl.height) for wl in wls], world)[rank]
        sub = ([raws[i] for i in mine], [params[i] for i in mine], [outs[i] for i in mine])
        ms_share = 0.0
        if mine:
            for _ in range(2):
                conv.demosaic_batch(*sub, stream=stream, graph=True)
            stream.synchronize()
            e0.record(stream)
            for _ in range(reps):
                conv.demosaic_batch(*sub, stream=stream, graph=True)
            e1.record(stream)
            stream.synchronize()
            ms_share = e0.elapsed_time(e1) / reps
    return {
        "workload": "16 frames: 4 x 4032x3024, 4 x 6000x4000, 4 x 5472x3648, 4 x 8368x5584, RGGB, 12/14-bit, "
                    "demosaic + 5-level denoise, FP16 storage",
        "megapixels_per_batch": mpix,
        "value": mpix / (ms_graph / 1e3),
        "unit": "MP/s",
        "ms_per_batch_graph": ms_graph,
        "ms_per_batch_stream_launched": ms_stream,
        "gpu_launches_per_batch": per_batch,
        "persistent": {"ms_per_batch_graph": ms_persistent, "value": mpix / (ms_persistent / 1e3), "unit": "MP/s",
                       "gpu_launches_per_batch": per_batch_persistent,
                       "note": "GLS_PERSISTENT + GLS_GRAPH: per frame the front end and the pyramid images, then "
                               "one persistent launch running every level of every frame (reconstruct, covariance, "
                               "eigen-solve, block matching) from a device work list, then the output transforms"},
        "strong": {"frames_this_rank": mine, "ms_share": ms_share,
                   "note": "the one batch split over the ranks by pixel count (longest-processing-time); "
                           "value = batch MP / the slowest rank's share time"},
        "block_match_tile_heights": [list(t) for t in block_match_tiles()],
        "note": "one CUDA graph replay per batch; frames spread largest-first over 6 slot streams; "
                "block_match_tile_heights: autotuned (width, height, variant = 10 x thread rows + pixels per thread: 84 and 162 are 32x32-pixel tiles, 44 and 82 are 32x16)",
    }


def post_leg(args, rank, local, conv, stream):
    """RawConverter::demosaic with postProcess on the headline workload: the
    six-frame (--post-frames) FP16 batch with GLS_POSTPROCESS (histogram statistics,
    guided-filter tone mapping, grain, sRGB tone curve) against the same
    batch without it, and the post-processing kernels' own device time per
    frame from the per-launch event profile. Roofline: the HBM bytes the
    post-processing must move per frame (denoised level 0 and the gradient in,
    RGBA FP16 out; FP16 planes) over its device time."""
    import torch

    import glasscamerapublic_b200 as g
    from glasscamerapublic_b200 import scene

    wl = scene.WORKLOADS[args.workload]
    params = scene.make_params(wl)
    H, W = wl.height, wl.width
    B = max(1, args.post_frames)
    dev = f"cuda:{local}"
    raws = [torch.from_numpy(scene.make_raw(wl, frame=100 + rank * B + f)[0].view(np.int16)).to(dev)
            for f in range(B)]
    outs = [torch.empty((H, W, 4), dtype=torch.float16, device=dev) for _ in range(B)]
    plist = [params] * B
    lib = g.lib()

    def stats():
        st = (g.KernelStat * 32)()
        n = C.c_int32()
        g.check(lib.gls_converter_stats(conv.handle, st, 32, C.byref(n)))
        return {st[i].name.decode(): {"launches": int(st[i].launches), "ms": st[i].ms} for i in range(n.value)}

    def batch_ms(post: bool) -> float:
        for _ in range(2):
            conv.demosaic_batch(raws, plist, outs, fp16=True, out_fp16=True, stream=stream, postProcess=post)
        stream.synchronize()
        reps = max(3, args.steps // 2)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            conv.demosaic_batch(raws, plist, outs, fp16=True, out_fp16=True, stream=stream, postProcess=post)
        e1.record(stream)
        stream.synchronize()
        return e0.elapsed_time(e1) / reps

    with torch.cuda.stream(stream):
        ms_plain = batch_ms(False)
        ms_post = batch_ms(True)
        g.check(lib.gls_converter_reset_stats(conv.handle))
        g.check(lib.gls_converter_set_profiling(conv.handle, 1))
        for i in range(B):
            conv.demosaic(raws[i], params, noiseReduction=True, fp16=True, out=outs[i], out_fp16=True,
                          stream=stream, sync=False, postProcess=True)
        stream.synchronize()
        pk = stats()["post_process"]
        g.check(lib.gls_converter_set_profiling(conv.handle, 0))
    post_ms = pk["ms"] / B
    px = W * H
    small = sum((W >> l) * (H >> l) for l in (2, 3, 4)) * 8  # levels 2, 3, 4 (FP16 RGBA)
    bytes_frame = px * (8 + 4 + 8) + small
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    gbs = bytes_frame / (post_ms / 1e3) / 1e9
    return {
        "workload": f"{B} x {W}x{H} RGGB 12-bit, demosaic + 5-level denoise + post-processing, FP16 storage",
        "value": B / (ms_post / 1e3), "unit": "frames/s",
        "ms_per_batch_post": ms_post, "ms_per_batch_plain": ms_plain,
        "added_ms_per_frame": (ms_post - ms_plain) / B,
        "post_kernels_ms_per_frame": post_ms,
        "post_launches_per_frame": pk["launches"] / B,
        "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                     "bytes_per_frame": bytes_frame,
                     "note": "all post-processing kernels of a frame together; bytes: denoised level 0 (8 B/px) "
                             "and gradient (4 B/px) read, RGBA FP16 (8 B/px) written, levels 2-4; peak "
                             + ("of measured" if peaks else "of fallback")},
    }


def calibrate_leg(args, rank, local, conv, stream):
    """RawConverter with calibrateFromImage on the headline workload: one
    12 MP frame at a time on the FP16 path, the raw noise model measured on
    the scaled frame and each of the five pyramid levels' models measured
    before the denoise (statistics kernels, then the two-pass FP64 fits on
    the device, each model read back to the host as the reference's host
    regressions return it), against the same frames through a converter
    that takes the calibration's models. Roofline: the HBM bytes the
    measurement moves per frame (statistics written once, read by each of
    the four fit passes) over its device time."""
    import torch

    import glasscamerapublic_b200 as g
    from glasscamerapublic_b200 import scene

    wl = scene.WORKLOADS[args.workload]
    params = scene.make_params(wl)
    H, W = wl.height, wl.width
    dev = f"cuda:{local}"
    # neutral step charts, the captures a noise model is measured on
    raws = [torch.from_numpy(scene.make_chart_raw(wl, frame=200 + rank * 2 + f)[0].view(np.int16)).to(dev)
            for f in range(2)]
    out = torch.empty((H, W, 4), dtype=torch.float16, device=dev)
    cal = g.RawConverter(local, calibrateFromImage=True)
    lib = g.lib()

    def frame_ms(c, n):
        for i in range(2):
            c.demosaic(raws[i % 2], params, fp16=True, out=out, out_fp16=True, stream=stream, sync=False)
        stream.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        for i in range(n):
            c.demosaic(raws[i % 2], params, fp16=True, out=out, out_fp16=True, stream=stream, sync=False)
        e1.record(stream)
        stream.synchronize()
        return max(e0.elapsed_time(e1), 1e3 * (time.perf_counter() - t0)) / n

    n = max(3, args.steps // 2)
    with torch.cuda.stream(stream):
        ms_plain = frame_ms(conv, n)
        ms_cal = frame_ms(cal, n)
        st = (g.KernelStat * 32)()
        k = C.c_int32()
        g.check(lib.gls_converter_reset_stats(cal.handle))
        g.check(lib.gls_converter_set_profiling(cal.handle, 1))
        for i in range(2):
            cal.demosaic(raws[i], params, fp16=True, out=out, out_fp16=True, stream=stream, sync=False)
        stream.synchronize()
        g.check(lib.gls_converter_stats(cal.handle, st, 32, C.byref(k)))
        nm = {st[i].name.decode(): (int(st[i].launches), st[i].ms) for i in range(k.value)}["noise_model"]
        g.check(lib.gls_converter_set_profiling(cal.handle, 0))
        (ra, rb), pyr = cal.noise_model()
    cal.close()
    nlf_ms = nm[1] / 2
    lv = [(W >> l) * (H >> l) for l in range(wl.levels)]
    q = (W // 2) * (H // 2)
    bytes_frame = (W * H * 2 + q * 32 + 3 * q * 32        # raw: scaled in, mean + var out, three fit passes
                   + sum(lv) * (8 + 16) + 3 * sum(lv) * 16)  # levels: FP16 in, statistics out, three fit passes
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    gbs = bytes_frame / (nlf_ms / 1e3) / 1e9
    return {
        "workload": f"{W}x{H} RGGB 12-bit step chart, demosaic + 5-level denoise, FP16 storage, calibrateFromImage",
        "value": 1e3 / ms_cal, "unit": "frames/s",
        "ms_per_frame_calibrating": ms_cal, "ms_per_frame_given_model": ms_plain,
        "measurement_ms_per_frame": nlf_ms, "measurement_launches_per_frame": nm[0] / 2,
        "measured_raw_b": [float(x) for x in rb], "given_raw_b": [float(params.raw_nlf.b[c]) for c in range(4)],
        "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                     "bytes_per_frame": bytes_frame,
                     "note": "all measurement kernels of a frame together (raw and five YCbCr levels: statistics "
                             "with the class histogram, then three fit passes each); peak "
                             + ("of measured" if peaks else "of fallback")},
        "note": "each measured model is read back to the host before the frame continues (six host syncs "
                "per frame), as the reference's host regressions are; frames run one at a time",
    }


def dng_leg(args, rank, local, conv, stream):
    """RawConverter::demosaic from DNG files, as pipelineTest's demosaicFile
    and PyramidFusion's runPipeline run it (pipelineTest.cpp:110-175,
    pyramidFusion.cpp:46-60): a 12 MP DNG with lossless-JPEG 256x256 tiles,
    as phone DNGs carry, read and decoded on the host's cores, parameters
    from its metadata and the camera calibration at its ISO, then demosaic,
    denoise and display post-processing on the GPU with the sRGB result back
    in host memory. Frames one at a time, wall clock."""
    import tempfile

    import glasscamerapublic_b200 as g
    from glasscamerapublic_b200 import dng, scene

    wl = scene.WORKLOADS[args.workload]
    tmp = tempfile.mkdtemp(prefix="gls_dng_")
    paths = []
    for f in range(2):
        raw, _ = scene.make_raw(wl, frame=300 + rank * 2 + f)
        info = g.DngInfo()
        info.cfa_pattern[:] = [0, 1, 1, 2]
        info.black_level, info.white_level, info.iso = wl.black, wl.white, wl.iso
        info.has_color_matrix2 = 1
        info.color_matrix2[:] = [0.66, -0.13, -0.07, -0.39, 1.21, 0.17, -0.06, 0.17, 0.55]
        info.has_as_shot_neutral = 1
        info.as_shot_neutral[:] = [0.52, 1.0, 0.61]
        info.make, info.model = b"Apple", b"iPhone 14 Pro"
        path = os.path.join(tmp, f"frame{f}.dng")
        dng.write_dng(path, raw, info, dng.COMPRESSION_LJ92, 256)
        paths.append(path)
    size = os.path.getsize(paths[0])

    def one(path):
        raw, info = dng.read_dng(path)
        p = dng.demosaic_params(info)
        return conv.demosaic(raw, p, fp16=True, out_fp16=True, postProcess=True)

    for path in paths:
        one(path)
    n = max(3, args.steps // 2)
    t0 = time.perf_counter()
    for i in range(n):
        out = one(paths[i % 2])
    t_frame = (time.perf_counter() - t0) / n
    # pipelined over files: the next file decoded on a host thread into a
    # pinned buffer while the GPU converts the current one
    seq = [paths[i % 2] for i in range(2 * n)]
    for _ in dng.convert_files(conv, paths):
        pass
    t0 = time.perf_counter()
    for _ in dng.convert_files(conv, seq):
        pass
    t_pipe = (time.perf_counter() - t0) / len(seq)
    t0 = time.perf_counter()
    for i in range(n):
        dng.read_dng(paths[i % 2])
    t_read = (time.perf_counter() - t0) / n
    for path in paths:
        os.remove(path)
    os.rmdir(tmp)
    return {
        "workload": f"{wl.width}x{wl.height} RGGB 12-bit DNG, lossless JPEG 256x256 tiles, "
                    "demosaic + 5-level denoise + post-processing, FP16 storage",
        "value": 1.0 / t_pipe, "unit": "frames/s",
        "ms_per_frame": 1e3 * t_pipe, "ms_per_frame_one_at_a_time": 1e3 * t_frame,
        "read_ms_per_frame": 1e3 * t_read,
        "decode_mp_per_s": wl.width * wl.height / 1e6 / t_read, "file_mb": size / 1e6,
        "host_threads": os.cpu_count(), "output": list(out.shape),
        "note": "wall clock per file: DNG read and lossless-JPEG decode on the host (tiles in parallel), "
                "parameters from the metadata, the GPU path with host I/O (FP16 sRGB out); value: files "
                "pipelined (dng.convert_files: the next file decoded into pinned memory while the GPU "
                "converts the current one); ms_per_frame_one_at_a_time: read, then convert, per file",
    }


def run_reference(args, rank):
    """The reference arm: the reference's path on the host cores, rank 0
    only. The Metal runtime cannot run here; the reference's own kernel
    source and camera calibration, compiled for the CPU (oracle/_ref),
    stand in for it, else the oracle port. A step is one full-resolution
    tile (1/16) of the 12 MP frame, the tiles taken in turn, so every 16
    steps cover one whole frame; frames/s = 1 / (16 x time per step). After
    the timed steps one whole 4032x3024 frame is converted once, untimed by
    the step clock, to check that 16 tiles take the time of a frame."""
    if rank != 0:
        return
    from glasscamerapublic_b200 import scene
    wl = scene.WORKLOADS[WORKLOAD]
    run_tile, run_frame, kind, what, threads, (tw, th) = cpu_frame_setup(wl)
    for i in range(args.warmup):
        run_tile(i)
    times = []
    for i in range(args.steps):
        t0 = time.perf_counter()
        run_tile(args.warmup + i)
        times.append(time.perf_counter() - t0)
    ms_step = 1e3 * sum(times) / len(times)
    v = 1e3 / (ms_step * TILES * TILES)
    full = None
    if not args.no_full_frame:
        t0 = time.perf_counter()
        run_frame()
        full = time.perf_counter() - t0
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f16/f32 (the reference's half/float kernels)",
            "data": "synthetic", "config": main_config(wl, args.gpus),
            "step": f"one {tw}x{th} full-resolution tile (1/{TILES * TILES}) of the {wl.width}x{wl.height} frame "
                    f"through the reference's demosaic + 5-level pyramid denoise; tiles in turn",
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": f"{args.steps} timed tiles of {tw}x{th}, {what}"},
            "full_frame": None if full is None else {
                "seconds": full, "frames_per_s": 1.0 / full,
                "tiles_equivalent_s": ms_step * TILES * TILES / 1e3,
                "note": "one whole 4032x3024 frame through the same code, timed once after the steps"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def bm_dram_traffic(wl):
    """DRAM bytes (read + write) of one frame's block-matching launches, from
    the committed ncu capture of the default matcher on the 4032x3024
    5-level workload (profiles/block_match_pair_dram_4032x3024.txt); None
    for other workloads."""
    f = Path(__file__).resolve().parent / "profiles" / "block_match_pair_dram_4032x3024.txt"
    if (wl.width, wl.height, wl.levels) != (4032, 3024, 5) or not f.exists():
        return None
    vals = {}
    for line in f.read_text().splitlines():
        if "=" in line and line.split("=")[0].strip() in ("traffic_bytes_per_frame", "algorithmic_bytes_per_frame"):
            vals[line.split("=")[0].strip()] = int(line.split("=")[1])
    if "traffic_bytes_per_frame" not in vals:
        return None
    return {"bytes": vals["traffic_bytes_per_frame"],
            "note": "dram__bytes_read.sum + dram__bytes_write.sum of one frame's 5 block-matching launches (one ncu "
                    "capture, profiles/block_match_pair_dram_4032x3024.txt), per frame like achieved; algorithmic "
                    f"bytes per frame {vals.get('algorithmic_bytes_per_frame')}"}


def main_config(wl, world, frames=N_ROTATE):
    """The workload description shared by both arms' lines."""
    return {"workload": wl.name, "frame": f"{wl.width}x{wl.height} RGGB 12-bit", "levels": wl.levels,
            "iso": wl.iso, "frames_per_step": frames,
            "l2": "each step reads 6 distinct frames; inputs + planes >> 126 MB L2",
            "parallelism": f"frames sharded over {world} rank(s), {frames}-frame batch per rank on 3 streams"}


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank)
        return
    import torch
    import torch.distributed as dist

    import glasscamerapublic_b200 as g
    from glasscamerapublic_b200 import scene

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()

    wl = scene.WORKLOADS[args.workload]
    params = scene.make_params(wl)
    conv = g.RawConverter(local)
    lib = g.lib()
    stream = torch.cuda.Stream()
    if (args.burst_only or args.adjoint_only or args.mixed_only or args.post_only or args.calibrate_only
            or args.dng_only):
        leg = (burst_leg if args.burst_only else adjoint_leg if args.adjoint_only else
               mixed_leg if args.mixed_only else post_leg if args.post_only else
               calibrate_leg if args.calibrate_only else dng_leg)
        b = leg(args, rank, local, conv, stream)
        if rank == 0:
            print(json.dumps({leg.__name__: True, **b}), flush=True)
        conv.close()
        if world > 1:
            dist.destroy_process_group()
        return
    H, W = wl.height, wl.width
    B = args.frames  # frames per step (one batch)

    # resident inputs: distinct frames per rank (weak scaling)
    made = [scene.make_raw(wl, frame=rank * B + f) for f in range(B)]
    raws_host = [m[0] for m in made]
    clean0 = made[0][1]
    del made
    raws = [torch.from_numpy(r.view(np.int16)).to(f"cuda:{local}") for r in raws_host]
    outs = [torch.empty((H, W, 4), dtype=torch.float16, device=f"cuda:{local}") for _ in range(B)]
    plist = [params] * B

    def step_batch():
        conv.demosaic_batch(raws, plist, outs, fp16=True, out_fp16=True, stream=stream)

    def step_frame(i, fp16=True, host_pca=False):
        conv.demosaic(raws[i % B], params, noiseReduction=True, fp16=fp16, out=outs[i % B], out_fp16=True,
                      stream=stream, host_pca=host_pca, sync=False)

    def stats():
        st = (g.KernelStat * 32)()
        n = C.c_int32()
        g.check(lib.gls_converter_stats(conv.handle, st, 32, C.byref(n)))
        return {st[i].name.decode(): {"launches": int(st[i].launches), "ms": st[i].ms} for i in range(n.value)}

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step_batch()
        stream.synchronize()
        g.check(lib.gls_converter_reset_stats(conv.handle))
        barrier()
        torch.cuda.synchronize()
        sampler = ClockSampler(local)
        sampler.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step_batch()
        e1.record(stream)
        stream.synchronize()
        clocks = sampler.stop()
        ms = e0.elapsed_time(e1)
        launches = sum(v["launches"] for v in stats().values())
        barrier()
        if args.quick:
            if rank == 0:
                print(json.dumps({"quick": True, "workload": args.workload, "frames_per_step": B,
                                  "ms_per_frame": ms / args.steps / B, "gpu_launches": launches}), flush=True)
            conv.close()
            if world > 1:
                dist.destroy_process_group()
            return

        # per-kernel device time: the same frames one after the other, each
        # launch bracketed by events on its stream
        g.check(lib.gls_converter_reset_stats(conv.handle))
        g.check(lib.gls_converter_set_profiling(conv.handle, 1))
        n_prof = max(B, args.steps)
        for i in range(n_prof):
            step_frame(i)
        per_kernel = stats()
        g.check(lib.gls_converter_set_profiling(conv.handle, 0))

        # FP32 plain single-frame path (FP32 planes, per-level host PCA sync:
        # the reference's structure)
        for i in range(2):
            step_frame(i, fp16=False, host_pca=True)
        stream.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n32 = max(3, args.steps // 2)
        f0.record(stream)
        for i in range(n32):
            step_frame(i, fp16=False, host_pca=True)
        f1.record(stream)
        stream.synchronize()
        ms32 = f0.elapsed_time(f1) / n32

        # end to end through the public batched call with host buffers
        # (pinned raw in, FP16 RGBA out; copies inside the timed region)
        pinned_raw = [torch.from_numpy(r.view(np.int16)).pin_memory() for r in raws_host]
        pinned_out = [torch.empty((H, W, 4), dtype=torch.float16).pin_memory() for _ in range(B)]

        def e2e_time(graph: bool) -> float:
            """ms per batch call; each call returns with the outputs in host
            memory. graph: the recorded batch (copies included) replayed."""
            def e2e_step():
                conv.demosaic_batch(pinned_raw, plist, pinned_out, fp16=True, out_fp16=True, stream=stream,
                                    graph=graph)

            e2e_step()
            e2e_step()
            n_e2e = max(3, args.steps // 2)
            barrier()
            t0 = time.perf_counter()
            g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            g0.record(stream)
            for _ in range(n_e2e):
                e2e_step()
            g1.record(stream)
            stream.synchronize()
            e2e_wall = (time.perf_counter() - t0) / n_e2e
            return max(g0.elapsed_time(g1) / n_e2e, 1e3 * e2e_wall)

        e2e_stream_ms = e2e_time(False)
        e2e_ms = e2e_time(True)

    # max over ranks
    from glasscamerapublic_b200.shard import max_over_ranks
    ms, ms32, e2e_ms, e2e_stream_ms = max_over_ranks([ms, ms32, e2e_ms, e2e_stream_ms], dist if world > 1 else None)
    ms_step = ms / args.steps
    value = world * B * args.steps / (ms / 1e3)

    # roofline of the dominant kernel (block matching) from the live event times
    bm = per_kernel.get("block_match", {"launches": 1, "ms": float("nan")})
    traffic = bm_dram_traffic(wl) if os.environ.get("GLS_BM_KERNEL", "") != "mma" else None
    px = sum((W >> i) * (H >> i) for i in range(wl.levels))
    taps = 21 * 21
    flop_per_tap = 50.0  # 8-D distance 24, chroma 6, two weights 8, accumulate 10 (FMA = 2)
    bm_tflops = px * taps * flop_per_tap * n_prof / (bm["ms"] / 1e3) / 1e12
    sm_clock = clocks.get("sm_mhz") or 1965.0
    fp32_peak = 148 * 128 * 2 * (sm_clock * 1e6) / 1e12  # SIMT FP32 FMA peak at the sampled clock
    mufu_rate = 148 * 16 * (sm_clock * 1e6) / 1e12       # ex2 per SM per clock = 16
    bm_mufu = px * taps * 2 * n_prof / (bm["ms"] / 1e3) / 1e12
    total_prof_ms = sum(v["ms"] for v in per_kernel.values())

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f16-storage/f32-math", "data": "synthetic",
        "config": main_config(wl, world, B),
        "e2e": {"value": world * B / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": B * W * H * 2,
                "d2h_bytes_per_step": B * W * H * 8,
                "stream_launched_value": world * B / (e2e_stream_ms / 1e3),
                "note": "gls_demosaic_batch with pinned host buffers (GLS_HOST_IO), returning with the FP16 RGBA "
                        "outputs in host memory; value: the recorded batch replayed (GLS_GRAPH, copies in the "
                        "graph); stream_launched_value: the same call without GLS_GRAPH"},
        "fp32_plain": {"value": world / (ms32 / 1e3), "unit": UNIT, "ms_per_frame": ms32,
                       "note": "FP32 planes, one frame at a time, per-level host PCA sync (the reference's structure)"},
        "speedup_vs_fp32_plain": ms32 / (ms_step / B),
        "roofline": {"bound": "fp32+mufu", "kernel": "block_match",
                     "achieved": bm_tflops, "peak": fp32_peak, "unit": "TFLOP/s", "frac": bm_tflops / fp32_peak,
                     "mufu_frac": bm_mufu / mufu_rate,
                     "traffic": traffic["bytes"] if traffic else None,
                     "traffic_note": traffic["note"] if traffic else "no DRAM capture for this matcher",
                     "share": bm["ms"] / total_prof_ms if total_prof_ms else None,
                     "ms_per_launch": bm["ms"] / max(1, bm["launches"]),
                     "peak_note": "nominal SIMT FP32 (148 SMs x 128 lanes x 2 x sampled SM clock); "
                                  "MEASURED_PEAKS has HBM and bf16-tensor peaks only"},
        "per_kernel_ms_per_frame": {k: v["ms"] / n_prof for k, v in per_kernel.items() if v["launches"]},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if not args.no_burst:
        b = burst_leg(args, rank, local, conv, stream)
        (b["ms_per_burst"],) = max_over_ranks([b["ms_per_burst"]], dist if world > 1 else None)
        line["burst"] = b
    if not args.no_mixed:
        mx = mixed_leg(args, rank, local, conv, stream)
        (mx["ms_per_batch_graph"],) = max_over_ranks([mx["ms_per_batch_graph"]], dist if world > 1 else None)
        mx["value"] = world * mx["megapixels_per_batch"] / (mx["ms_per_batch_graph"] / 1e3)
        mx["scaling"] = "weak: every rank converts the whole batch"
        (mx["strong"]["ms_share"],) = max_over_ranks([mx["strong"]["ms_share"]], dist if world > 1 else None)
        mx["strong"]["value"] = mx["megapixels_per_batch"] / (mx["strong"]["ms_share"] / 1e3)
        mx["strong"]["unit"] = "MP/s"
        line["mixed_batch"] = mx
    if not args.no_post:
        pp = post_leg(args, rank, local, conv, stream)
        (pp["ms_per_batch_post"],) = max_over_ranks([pp["ms_per_batch_post"]], dist if world > 1 else None)
        pp["value"] = world * max(1, args.post_frames) / (pp["ms_per_batch_post"] / 1e3)
        line["post_process"] = pp
    if not args.no_dng:
        dl = dng_leg(args, rank, local, conv, stream)
        (dl["ms_per_frame"],) = max_over_ranks([dl["ms_per_frame"]], dist if world > 1 else None)
        dl["value"] = world * 1e3 / dl["ms_per_frame"]
        line["dng_file"] = dl
    if not args.no_calibrate:
        cl = calibrate_leg(args, rank, local, conv, stream)
        (cl["ms_per_frame_calibrating"],) = max_over_ranks([cl["ms_per_frame_calibrating"]],
                                                           dist if world > 1 else None)
        cl["value"] = world * 1e3 / cl["ms_per_frame_calibrating"]
        line["calibrate"] = cl
    if not args.no_adjoint:
        a = adjoint_leg(args, rank, local, conv, stream)
        (a["ms_per_batch"],) = max_over_ranks([a["ms_per_batch"]], dist if world > 1 else None)
        line["adjoint"] = a
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # one frame's error against the FP64 oracle, through the same calls
        # as the timed paths (batched FP16, plain FP32 with host PCA)
        o16 = np.empty((H, W, 4), np.float16)
        conv.demosaic_batch([raws_host[0]], [params], [o16], fp16=True, out_fp16=True, sync=True)
        o32 = conv.demosaic(raws_host[0], params, noiseReduction=True, fp16=False, host_pca=True)
        line["error_vs_fp64"] = fp64_check_leg(wl, raws_host[0], clean0, o16.astype(np.float32), o32)
        line["cpu_baseline"] = cpu_baseline(wl, args.cpu_seconds)
    if rank == 0:
        print(json.dumps(line), flush=True)
    conv.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
