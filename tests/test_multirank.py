"""Multi-rank host logic on CPU: frame sharding, the max-over-ranks
timing reduction and the data-parallel calibration gradient all-reduce,
run as two gloo ranks (no GPU)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import numpy as np

from glasscamerapublic_b200.shard import assign_frames, max_over_ranks, mean_gradient
from glasscamerapublic_b200 import scene


def test_assign_frames_covers_every_frame_once_and_balances():
    sizes = [(wl.width, wl.height) for wl in scene.mixed_batch()]  # the 16-frame mixed-sensor batch
    for world in (1, 2, 4, 8):
        parts = assign_frames(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i][0] * sizes[i][1] for i in p) for p in parts]
        biggest = max(w * h for w, h in sizes)
        assert max(loads) - min(loads) <= biggest
    assert assign_frames([(4, 4)] * 3, 2) == [[0, 2], [1]]
    with pytest.raises(ValueError):
        assign_frames(sizes, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sizes = [(wl.width, wl.height) for wl in scene.mixed_batch()]
        mine = assign_frames(sizes, world)[rank]
        # each rank "times" its share; the job time is the max over ranks
        fake_ms = [float(sum(sizes[i][0] * sizes[i][1] for i in mine)) / 1e6, float(rank + 1)]
        out = max_over_ranks(fake_ms, dist)
        # calibration: rank r holds r + 1 frames whose gradients are all (r + 1)
        nf = rank + 1
        gsum = np.full(32, float(rank + 1)) * nf
        gm = mean_gradient(gsum, nf, dist)
        q.put((rank, mine, out, gm.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    (r0, m0, o0, g0), (r1, m1, o1, g1) = res
    assert sorted(m0 + m1) == list(range(16)) and not set(m0) & set(m1)
    # mean over the 3 frames: (1 * 1 + 2 * 2) / 3, identical on both ranks
    assert g0 == g1 and np.allclose(g0, 5.0 / 3.0)
    assert o0 == o1  # both ranks see the same reduced timings
    sizes = [(wl.width, wl.height) for wl in scene.mixed_batch()]
    loads = [sum(sizes[i][0] * sizes[i][1] for i in m) / 1e6 for m in (m0, m1)]
    assert o0[0] == pytest.approx(max(loads)) and o0[1] == 2.0


def test_mean_gradient_without_a_process_group():
    assert np.allclose(mean_gradient(np.arange(4.0) * 2, 2), np.arange(4.0))


def test_burst_members_cover_the_burst():
    from glasscamerapublic_b200.shard import burst_members
    for n in (1, 4, 8):
        for world in (1, 2, 3, 4, 8):
            parts = burst_members(n, world)
            assert len(parts) == world and 0 in parts[0]
            assert sorted(m for p in parts for m in p) == list(range(n))
    assert burst_members(4, 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        burst_members(4, 0)


def _burst_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from glasscamerapublic_b200 import KEYPOINT_DTYPE, shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(7)
        kps = np.zeros(37, KEYPOINT_DTYPE)
        kps.view(np.float32).reshape(37, -1)[:] = rng.normal(size=(37, KEYPOINT_DTYPE.itemsize // 4))
        desc = rng.normal(size=(37, 64)).astype(np.float32)
        # rank 0 holds the features and the header; the others pass nothing
        kb, db = shard.broadcast_features(kps if rank == 0 else np.zeros(0, KEYPOINT_DTYPE),
                                          desc if rank == 0 else np.zeros((0, 64), np.float32), dist)
        head = shard.broadcast_bytes(b"params:" + bytes(range(200)) if rank == 0 else None, dist)
        empty = shard.broadcast_bytes(b"" if rank == 0 else None, dist)
        # homographies: member m > 0 of rank m % world fills row m - 1
        members = [m for m in shard.burst_members(4, world)[rank] if m > 0]
        rows = np.array([np.full(9, 10.0 * m + 0.5) for m in members], np.float32).reshape(-1, 9)
        Hall = shard.all_gather_rows(rows, [m - 1 for m in members], 3, dist)
        # running means of warped members: member m's frame is the constant m
        part = torch.full((4, 6, 4), float(np.mean(members)) if members else 0.0)
        mean = shard.reduce_mean(part, len(members), 3, dist)
        q.put((rank, kb.numpy().tobytes() == kps.tobytes(), np.array_equal(db.numpy(), desc), head, empty,
               Hall.tolist(), None if mean is None else mean.numpy().tolist()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_split_a_burst(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_burst_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want_H = [[10.0 * m + 0.5] * 9 for m in (1, 2, 3)]
    for rank, k_ok, d_ok, head, empty, Hall, mean in res:
        assert k_ok and d_ok
        assert head == b"params:" + bytes(range(200)) and empty == b""
        assert Hall == want_H
        if rank == 0:
            assert np.allclose(mean, 2.0)  # the mean of members 1, 2, 3
        else:
            assert mean is None


def test_burst_helpers_without_a_process_group():
    import torch
    from glasscamerapublic_b200 import KEYPOINT_DTYPE, shard
    kps = np.zeros(3, KEYPOINT_DTYPE)
    kb, db = shard.broadcast_features(kps, np.ones((3, 64), np.float32))
    assert kb.numel() == 3 * KEYPOINT_DTYPE.itemsize and db.shape == (3, 64)
    assert shard.broadcast_bytes(b"abc") == b"abc"
    assert np.array_equal(shard.all_gather_rows(np.ones((2, 9)), [0, 2], 3), [[1] * 9, [0] * 9, [1] * 9])
    t = torch.ones(2, 2)
    assert shard.reduce_mean(t, 3, 3) is t


def _fake_burst_rank(rank, world, port, q):
    """fuse_burst_sharded's orchestration with the detector, the warps, the
    DNG reader and the converter replaced by CPU fakes whose outputs encode
    which frame (and which broadcast reference) they came from."""
    import types
    import torch
    import torch.distributed as dist
    import glasscamerapublic_b200 as g
    from glasscamerapublic_b200 import KEYPOINT_DTYPE, burst, dng, registration
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        def read_dng(path):
            m = int(str(path)[1:])
            info = types.SimpleNamespace(bayer_pattern=2, black_level=0, white_level=4095, baseline_exposure=0.0)
            return np.full((8, 12), 100 * m + 7, np.uint16), info

        class FakeSURF:
            def __init__(self, w, h, **kw):
                self.slots = {}

            def raw_channels(self, raw, pattern, black, white, exposure, outs=None, stream=None):
                outs[1].fill_(float(raw[0, 0]))
                outs[3].fill_(float(raw[0, 0]) + 0.5)

            def detect_slot(self, plane, slot, stream=None):
                v = float(plane[0, 0])
                k = np.zeros(3, KEYPOINT_DTYPE)
                k["x"] = v
                self.slots[slot] = (k, np.full((3, 64), v, np.float32))

            def features(self, slot, stream=None):
                return self.slots[slot]

            def load_features(self, slot, kps, desc, stream=None):
                self.slots[slot] = (np.array(kps).copy(), np.array(desc).copy())

            def register_frames(self, ref_slots, frame_slots, *a):
                out = []
                for f0, f1 in frame_slots:
                    H = np.eye(3, dtype=np.float32)
                    H[0, 2] = self.slots[f0][1][0, 0] - self.slots[ref_slots[0]][1][0, 0]
                    H[1, 2] = self.slots[f1][0]["x"][0] - self.slots[ref_slots[1]][0]["x"][0]
                    out.append(H)
                return np.array(out, np.float32).reshape(-1, 3, 3)

            def close(self):
                pass

        def fuse(fused, inp, out, H, count, stream=None):
            out.copy_(((count - 1) * fused + inp + float(H[0][2])) / count)

        def register_image(inp, out, H, stream=None):
            out.copy_(inp + float(H[0][2]))

        conv = types.SimpleNamespace(
            demosaic=lambda raw, p, fp16=True, postProcess=True: torch.full(
                (raw.shape[0], raw.shape[1], 4), float(raw[0, 0])))
        dng.read_dng = read_dng
        dng.demosaic_params = lambda info: g.DemosaicParams()
        registration.SURF = FakeSURF
        registration.RegisterAndFuseKernel = lambda: fuse
        registration.register_image = register_image
        written = []
        burst.write_tiff_rgb8 = lambda path, rgba, stream=None: written.append(str(path))
        fused, Hall, out = burst.fuse_burst_sharded(conv, ["f1", "f2", "f3", "f0"], dist, out_path="fused.tiff",
                                                    device="cpu")
        q.put((rank, Hall.tolist(), None if fused is None else fused.numpy().tolist(), out, written))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [1, 2, 5])
def test_burst_split_orchestration_with_more_ranks_than_frames(world):
    # world 5 > 4 frames: rank 4 holds nothing and rank 0 only the
    # reference, yet every rank takes the same collective steps
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_fake_burst_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want_H = [[[1.0, 0.0, 100.0 * m], [0.0, 1.0, 100.0 * m], [0.0, 0.0, 1.0]] for m in (1, 2, 3)]
    for rank, Hall, fused, out, written in res:
        assert Hall == want_H, rank
        if rank == 0:
            # member m's frame is 100 m + 7, warped by + 100 m: the mean of 207, 407, 607
            assert np.allclose(fused, 407.0) and out == "fused.tiff" and written == ["fused.tiff"]
        else:
            assert fused is None and out is None and written == []
