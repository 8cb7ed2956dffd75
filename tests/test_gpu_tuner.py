"""The calibration tuner on the GPU: its loss and gradient over several
frames are the mean of the adjoint's per-frame values, and a few Adam steps
from a miscalibrated start (denoise strengths at a quarter of the
calibration's) lower the mean loss against the clean targets."""
import numpy as np
import pytest

from glasscamerapublic_b200 import ADJ_CHROMA, ADJ_LUMA
from glasscamerapublic_b200 import adjoint as A
from glasscamerapublic_b200 import scene
from glasscamerapublic_b200.tuner import CalibrationTuner

pytestmark = pytest.mark.gpu


def _frames(n):
    wl = scene.Workload("tune", 192, 128, levels=3, gain=0.8, read=3.0, iso=1600, seed=90)
    raws, targets = [], []
    for f in range(n):
        raw, clean = scene.make_raw(wl, f)
        raws.append(raw)
        targets.append(scene.target_rgb(clean).astype(np.float32))
    return wl, raws, targets


def test_tuner_mean_matches_per_frame_adjoint(converter):
    wl, raws, targets = _frames(3)
    p = scene.make_params(wl)
    tun = CalibrationTuner.for_frames(converter, raws, targets, p)
    loss, grad = tun.evaluate()
    per = [A.loss_and_grad(converter, r, p, t) for r, t in zip(raws, targets)]
    assert loss == pytest.approx(np.mean([l for l, _ in per]), rel=1e-12)
    assert np.allclose(grad, np.mean([g.astype(np.float64) for _, g in per], axis=0), rtol=1e-12, atol=0)
    # one process holds the whole job: for_job takes every frame
    lj, gj = CalibrationTuner.for_job(converter, raws, targets, p).evaluate()
    assert lj == loss and np.array_equal(gj, grad)


def test_tuner_lowers_the_loss_from_a_miscalibrated_start(converter, tmp_path):
    wl, raws, targets = _frames(2)
    good = scene.make_params(wl)
    th = A.params_to_theta(good)
    for l in range(wl.levels):
        th[ADJ_LUMA + l] *= 0.25
        th[ADJ_CHROMA + l] *= 0.25
    start = A.theta_to_params(th, good)
    tun = CalibrationTuner.for_frames(converter, raws, targets, start, lr=0.1)
    losses = tun.run(8, checkpoint=tmp_path / "t.json")
    final, _ = tun.evaluate()
    assert final < 0.97 * losses[0], (losses, final)
    # the finest level's luma strength moved up, towards the calibration
    # (on these synthetic scenes the chroma optimum lies below the start)
    assert tun.theta[ADJ_LUMA] > th[ADJ_LUMA]
    # the tuned parameters run through the forward path
    out = tun.params()
    assert out.denoise[0].luma == pytest.approx(tun.theta[ADJ_LUMA])
