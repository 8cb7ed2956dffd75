"""The hand-written adjoint (gls_demosaic_denoise_vjp) against the reference
gradient: torch.autograd of the float64 re-expression of the pyramid
(tests/_torch_pyramid.py, itself checked against central differences of the
FP64 oracle), fed the CUDA forward's own despeckled image, gradient plane and
PCA bases. The adjoint runs in FP32; tolerances:
  * loss: 1e-4 relative;
  * each gradient entry of at least 1e-2 of the largest entry of its
    parameter kind (per-level luma, chroma, A_Y, B_Y, A_C, B_C): 1e-3
    relative; every entry: 1e-3 of its magnitude plus 1e-5 of the largest
    entry of its kind, which absorbs FP32 rounding on near-zero entries
    (the coarsest levels' entries can be 1e-12 of the finest's);
  * dL/d(despeckled image), per pixel: 1e-3 of its largest entry.
The full-size case (one 2048x1536 frame of the calibration workload) runs
the float64 reference on the GPU, its window rows checkpointed.
The raw-green entries (30, 31) act through the front end: they are checked
against central differences of the loss, the front end run by the FP64
oracle's stages and the pyramid by the oracle's FP64 pyramid with the same
fixed bases and gradient plane: 2% of the magnitude plus 1% of the larger."""
import numpy as np
import pytest
import torch

import _oracle as O
import _torch_pyramid as TP
import glasscamerapublic_b200 as g
from glasscamerapublic_b200 import adjoint as A
from glasscamerapublic_b200 import scene

pytestmark = pytest.mark.gpu


def _reference(converter, p, target, levels, device="cpu", checkpoint=False):
    ds = converter.plane(g.PLANE_DESPECKLED)
    grad = converter.plane(g.PLANE_GRADIENT)
    bases = np.stack([converter.pca_basis(l) for l in range(levels)]).astype(np.float64)
    _, inv = O.cam_ycbcr(np.eye(3), scene.XYZ_SRGB)
    return TP.loss_and_grad(ds, grad, p, bases, inv, target, device=device, checkpoint=checkpoint)


def _check(loss, grad, loss_t, g_t, levels):
    assert abs(loss - loss_t) <= 1e-4 * loss_t, (loss, loss_t)
    assert np.all(np.isfinite(grad))
    for kind in range(6):
        sl = slice(5 * kind, 5 * kind + levels)
        ref = g_t[sl]
        got = grad[sl].astype(np.float64)
        big = np.abs(ref) >= 1e-2 * np.abs(ref).max()
        assert np.all(np.abs(got - ref)[big] <= 1e-3 * np.abs(ref)[big]), (kind, got, ref)
        tol = 1e-3 * np.abs(ref) + 1e-5 * np.abs(ref).max() + 1e-30
        assert np.all(np.abs(got - ref) <= tol), (kind, got, ref)
        assert np.all(grad[5 * kind + levels:5 * kind + 5] == 0)


@pytest.mark.parametrize("levels,iso,size", [(3, 400, (160, 96)), (4, 1600, (192, 128))])
def test_adjoint_matches_autograd(converter, levels, iso, size):
    w, h = size
    wl = scene.Workload("adj", w, h, levels=levels, gain=0.8, read=3.0, iso=iso, seed=30 + levels)
    raw, clean = scene.make_raw(wl)
    p = scene.make_params(wl)
    target = scene.target_rgb(clean).astype(np.float32)
    loss, grad = A.loss_and_grad(converter, raw, p, target)
    loss_t, g_t, _ = _reference(converter, p, target, levels)
    _check(loss, grad, loss_t, g_t, levels)


def test_adjoint_full_size_calibration_frame(converter):
    # one frame of the 8 x 2048x1536 calibration workload, 5 levels
    wl = scene.Workload("cfg5_2048x1536", 2048, 1536, levels=5, gain=1.0, read=4.0, iso=800, seed=5000)
    raw, clean = scene.make_raw(wl)
    p = scene.make_params(wl)
    target = scene.target_rgb(clean).astype(np.float32)
    loss, grad = A.loss_and_grad(converter, raw, p, target)
    loss_t, g_t, _ = _reference(converter, p, target, 5, device="cuda", checkpoint=True)
    torch.cuda.empty_cache()
    _check(loss, grad, loss_t, g_t, 5)


def test_adjoint_input_gradient_matches_autograd(converter):
    # dL/d(despeckled image): the pyramid's reverse sweep down to its input,
    # which the raw-green entries build on
    wl = scene.Workload("adj", 160, 112, levels=3, gain=0.8, read=3.0, iso=800, seed=61)
    raw, clean = scene.make_raw(wl)
    p = scene.make_params(wl)
    target = scene.target_rgb(clean).astype(np.float32)
    A.loss_and_grad(converter, raw, p, target)
    g_ds = converter.plane(g.PLANE_ADJ_DESPECKLED)
    ds = converter.plane(g.PLANE_DESPECKLED)
    grad = converter.plane(g.PLANE_GRADIENT)
    bases = np.stack([converter.pca_basis(l) for l in range(3)]).astype(np.float64)
    _, inv = O.cam_ycbcr(np.eye(3), scene.XYZ_SRGB)
    *_, g_ref = TP.loss_and_grad(ds, grad, p, bases, inv, target, with_ds=True)
    assert g_ds.shape == g_ref.shape
    assert np.abs(g_ds - g_ref).max() <= 1e-3 * np.abs(g_ref).max()


def _front_loss(raw, p, grad, bases, inv, target):
    """The loss with the front end from the FP64 oracle's stages and the
    pyramid from the FP64 oracle (bases and gradient plane fixed)."""
    h, w = raw.shape
    s = O.stage("scale", p=p, w=w, h=h, out_shape=(h, w), raw=raw, f64=True)
    if p.high_noise_image:
        s = O.stage("raw_denoise", s, grad, p=p, w=w, h=h, out_shape=(h, w), f64=True)
    rgb = O.stage("demosaic_rgb", s, grad, p=p, w=w, h=h, out_shape=(h, w, 4), f64=True)
    fwd, _ = O.cam_ycbcr(np.eye(3), scene.XYZ_SRGB)
    ycc = np.zeros((h, w, 4), np.float32)
    ycc[..., :3] = rgb[..., :3].astype(np.float64) @ np.asarray(fwd, np.float64).T
    ds = O.stage("despeckle", ycc, p=p, w=w, h=h, out_shape=(h, w, 4), f64=True)
    return O.pyramid_loss(ds, grad, p, bases, inv, target)


@pytest.mark.parametrize("high_noise", [True, False])
def test_raw_green_gradient_matches_finite_differences(converter, high_noise):
    wl = scene.Workload("adj", 128, 96, levels=3, gain=0.6, read=4.0, iso=800, seed=71)
    raw, clean = scene.make_raw(wl)
    p = scene.make_params(wl)
    p.high_noise_image = 1 if high_noise else 0
    target = scene.target_rgb(clean).astype(np.float32)
    loss, grad = A.loss_and_grad(converter, raw, p, target)
    gplane = converter.plane(g.PLANE_GRADIENT)
    bases = np.stack([converter.pca_basis(l) for l in range(3)]).astype(np.float64)
    _, inv = O.cam_ycbcr(np.eye(3), scene.XYZ_SRGB)
    theta = A.params_to_theta(p)
    fd = []
    # steps on the scale of the green variance gv0 + gv1 * signal they enter
    steps = {30: 2e-3 * 0.2 * theta[31], 31: 2e-3 * theta[31]}
    for k in (30, 31):
        hstep = steps[k]
        lp = _front_loss(raw, A.theta_to_params(theta + hstep * np.eye(32)[k], p), gplane, bases, inv, target)
        lm = _front_loss(raw, A.theta_to_params(theta - hstep * np.eye(32)[k], p), gplane, bases, inv, target)
        fd.append((lp - lm) / (2 * hstep))
    fd = np.array(fd)
    big = np.abs(fd).max()
    assert big > 0
    assert np.all(np.abs(grad[30:32] - fd) <= 0.02 * np.abs(fd) + 0.01 * big), (grad[30:32], fd)


def test_adjoint_device_inputs_and_autograd_function(converter):
    wl = scene.Workload("adj", 128, 96, levels=3, gain=0.8, read=3.0, iso=800, seed=40)
    raw, clean = scene.make_raw(wl)
    p = scene.make_params(wl)
    target = scene.target_rgb(clean).astype(np.float32)
    l0, g0 = A.loss_and_grad(converter, raw, p, target)
    rd = torch.from_numpy(raw.view(np.int16)).cuda()
    td = torch.from_numpy(target).cuda()
    l1, g1 = A.loss_and_grad(converter, rd, p, td)
    torch.cuda.synchronize()
    assert l0 == l1 and np.array_equal(g0, g1)
    # the autograd binding returns the same gradient
    F = A.denoise_loss_function()
    theta = torch.tensor(A.params_to_theta(p), dtype=torch.float64, requires_grad=True)
    loss = F.apply(theta, converter, raw, p, target)
    loss.backward()
    assert abs(float(loss.detach()) - l0) <= 1e-6 * l0
    assert np.allclose(theta.grad.numpy(), g0.astype(np.float64), rtol=1e-6, atol=0)


def test_pyramid_denoise_vjp_matches_autograd(converter):
    # the denoise-only VJP: a random cotangent of the denoised YCbCr
    wl = scene.Workload("adj", 160, 112, levels=3, gain=0.8, read=3.0, iso=800, seed=81)
    raw, _ = scene.make_raw(wl)
    p = scene.make_params(wl)
    converter.demosaic(raw, p)  # a realistic despeckled image and gradient
    ds = converter.plane(g.PLANE_DESPECKLED)
    grad = converter.plane(g.PLANE_GRADIENT)
    rng = np.random.default_rng(5)
    g_out = rng.standard_normal((112, 160, 4)).astype(np.float32) * 1e-3
    pp = g.PyramidProcessor(converter)
    gt, g_ycc = pp.denoise_vjp(ds, grad, p, g_out)
    bases = np.stack([converter.pca_basis(l) for l in range(3)]).astype(np.float64)
    g_ref, gds_ref = TP.vjp(ds, grad, p, bases, g_out)
    assert np.all(gt[30:] == 0) and np.all(gt[3:5] == 0)
    for kind in range(6):
        sl = slice(5 * kind, 5 * kind + 3)
        ref = g_ref[sl]
        tol = 1e-3 * np.abs(ref) + 1e-4 * np.abs(ref).max() + 1e-30  # a random cotangent: sums that cancel
        assert np.all(np.abs(gt[sl].astype(np.float64) - ref) <= tol), (kind, gt[sl], ref)
    assert np.abs(g_ycc - gds_ref).max() <= 1e-3 * np.abs(gds_ref).max()
