"""The calibration tuner's host logic on CPU: Adam with per-parameter
scales converges on a quadratic whose minimiser spans many decades, the
box keeps strengths positive, a checkpointed run resumes bit for bit, and
two gloo ranks holding different frames take the same steps as one process
holding all of them."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from glasscamerapublic_b200 import ADJ_LUMA, ADJ_NPARAMS
from glasscamerapublic_b200.tuner import AdamBox, CalibrationTuner, default_box


def _theta0():
    # magnitudes like a calibration: strengths ~1, NLF coefficients ~1e-5
    t = np.zeros(ADJ_NPARAMS)
    t[0:10] = np.linspace(0.5, 2.0, 10)
    t[10:30] = np.geomspace(1e-6, 1e-4, 20)
    t[30], t[31] = 2e-6, 3e-5
    return t


def _quadratic(target, weight):
    """Frame i's loss: sum weight * ((theta - target_i) / |target|)^2, with
    target_i = target * (1 + 0.01 i): the mean-loss minimiser is the mean
    of the frames' targets."""
    mag = np.abs(target)

    def grad_fn(theta, i):
        ti = target * (1 + 0.01 * i)
        r = (theta - ti) / mag
        return float(np.sum(weight * r * r)), 2 * weight * r / mag

    return grad_fn


def test_adam_converges_across_decades():
    t0 = _theta0()
    target = t0 * 1.3
    n = 4
    tun = CalibrationTuner(t0, _quadratic(target, np.ones(ADJ_NPARAMS)), n, lr=0.02)
    losses = tun.run(400)
    best = target * (1 + 0.01 * (n - 1) / 2)
    floor = np.mean([fn_loss for fn_loss, _ in (_quadratic(target, np.ones(ADJ_NPARAMS))(best, i)
                                              for i in range(n))])
    assert losses[-1] <= floor * (1 + 1e-6) and losses[0] > 100 * floor
    assert np.all(np.abs(tun.theta - best) <= 2e-3 * np.abs(best)), (tun.theta / best)


def test_box_keeps_strengths_positive_and_freezes_zeros():
    t0 = _theta0()
    t0[4] = 0.0  # a level the pyramid does not have
    target = t0.copy()
    target[ADJ_LUMA + 1] = -5.0  # pulls a strength below zero
    target[4] = 1.0
    mag = np.where(t0 != 0, np.abs(t0), 1.0)

    def grad_fn(theta, i):
        r = (theta - target) / mag
        return float(r @ r), 2 * r / mag

    tun = CalibrationTuner(t0, grad_fn, 1, lr=0.2)
    tun.run(200)
    _, lo, _ = default_box(t0)
    th = tun.theta
    assert th[ADJ_LUMA + 1] == pytest.approx(lo[ADJ_LUMA + 1]) and th[ADJ_LUMA + 1] > 0
    assert th[4] == 0.0
    assert np.all(th >= lo)


def test_checkpoint_resumes_bit_for_bit(tmp_path):
    t0 = _theta0()
    fn = _quadratic(t0 * 0.7, np.linspace(0.5, 1.5, ADJ_NPARAMS))
    whole = CalibrationTuner(t0, fn, 3, lr=0.05)
    whole.run(12)
    ck = tmp_path / "tuner.json"
    first = CalibrationTuner(t0, fn, 3, lr=0.05)
    first.run(5, checkpoint=ck, every=2)
    second = CalibrationTuner(np.ones(ADJ_NPARAMS), fn, 3)
    second.load(ck)
    assert second.opt.t == 5 and second.history == first.history
    second.run(7)
    assert np.array_equal(second.theta, whole.theta)
    assert second.history == whole.history
    assert not (tmp_path / "tuner.json.tmp").exists()
    with pytest.raises(ValueError):
        second.load_state_dict({"format": "something else"})


def test_non_finite_gradient_raises():
    t0 = _theta0()
    tun = CalibrationTuner(t0, lambda th, i: (float("nan"), np.zeros(ADJ_NPARAMS)), 1)
    with pytest.raises(FloatingPointError):
        tun.step()
    assert tun.opt.t == 0 and np.array_equal(tun.theta, t0)


def test_adam_state_round_trip():
    s, lo, hi = default_box(_theta0())
    a = AdamBox(_theta0(), s, lo, hi, lr=0.1)
    g = np.linspace(-1, 1, ADJ_NPARAMS)
    a.step(g)
    b = AdamBox.from_state(a.state())
    assert np.array_equal(a.step(g), b.step(g))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_worker(rank, world, port, ck, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t0 = _theta0()
        fn = _quadratic(t0 * 1.2, np.ones(ADJ_NPARAMS))
        mine = [0, 1, 2] if rank == 0 else [3, 4]  # unequal shares of five frames
        tun = CalibrationTuner(t0, lambda th, i: fn(th, mine[i]), len(mine), lr=0.05, dist=dist)
        tun.run(6, checkpoint=ck)
        q.put((rank, tun.theta.tolist(), tun.history))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_step_together(tmp_path):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ck = str(tmp_path / "dp.json")
    procs = [ctx.Process(target=_rank_worker, args=(r, 2, port, ck, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, th0, h0), (_, th1, h1) = res
    assert th0 == th1 and h0 == h1  # every rank takes the same step
    t0 = _theta0()
    single = CalibrationTuner(t0, _quadratic(t0 * 1.2, np.ones(ADJ_NPARAMS)), 5, lr=0.05)
    single.run(6)
    assert np.allclose(th0, single.theta, rtol=1e-12, atol=0)
    assert np.allclose(h0, single.history, rtol=1e-12)
    # rank 0 alone wrote the checkpoint, with the shared state
    back = CalibrationTuner(np.ones(ADJ_NPARAMS), None, 0)
    back.load(ck)
    assert back.theta.tolist() == th0


def test_job_share_without_a_process_group_is_every_frame():
    assert CalibrationTuner.job_share([(64, 48), (32, 24), (128, 96)]) == [0, 1, 2]


_JOB_SIZES = [(640, 480), (320, 240), (800, 600), (160, 120)]


def _share_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = CalibrationTuner.job_share(_JOB_SIZES, dist)
        t0 = _theta0()
        fn = _quadratic(t0 * 0.8, np.ones(ADJ_NPARAMS))
        tun = CalibrationTuner(t0, lambda th, i: fn(th, mine[i]), len(mine), lr=0.05, dist=dist)
        tun.run(4)
        q.put((rank, mine, tun.theta.tolist()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [3, 5])
def test_gloo_ranks_share_a_job(world):
    # five ranks over four frames: one rank holds none and still takes part
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_share_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(i for _, mine, _ in res for i in mine) == list(range(len(_JOB_SIZES)))
    assert all(th == res[0][2] for _, _, th in res)
    t0 = _theta0()
    single = CalibrationTuner(t0, _quadratic(t0 * 0.8, np.ones(ADJ_NPARAMS)), len(_JOB_SIZES), lr=0.05)
    single.run(4)
    assert np.allclose(res[0][2], single.theta, rtol=1e-12, atol=0)
