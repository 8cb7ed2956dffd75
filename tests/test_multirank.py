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
