"""The hand-written adjoint (gls_demosaic_denoise_vjp) against the reference
gradient: torch.autograd of the float64 re-expression of the pyramid
(tests/_torch_pyramid.py, itself checked against central differences of the
FP64 oracle), fed the CUDA forward's own despeckled image, gradient plane and
PCA bases. The adjoint runs in FP32; tolerances:
  * loss: 1e-4 relative;
  * each gradient entry: 2e-3 of its magnitude plus 1e-3 of the largest
    entry of the same parameter kind (per-level luma, chroma, A_Y, B_Y,
    A_C, B_C), which absorbs FP32 rounding on near-zero entries."""
import numpy as np
import pytest
import torch

import _oracle as O
import _torch_pyramid as TP
import glasscamerapublic_b200 as g
from glasscamerapublic_b200 import adjoint as A
from glasscamerapublic_b200 import scene

pytestmark = pytest.mark.gpu


def _reference(converter, p, target, levels):
    ds = converter.plane(g.PLANE_DESPECKLED)
    grad = converter.plane(g.PLANE_GRADIENT)
    bases = np.stack([converter.pca_basis(l) for l in range(levels)]).astype(np.float64)
    _, inv = O.cam_ycbcr(np.eye(3), scene.XYZ_SRGB)
    return TP.loss_and_grad(ds, grad, p, bases, inv, target)


def _check(loss, grad, loss_t, g_t, levels):
    assert abs(loss - loss_t) <= 1e-4 * loss_t, (loss, loss_t)
    assert np.isnan(grad[30]) and np.isnan(grad[31])
    for kind in range(6):
        sl = slice(5 * kind, 5 * kind + levels)
        ref = g_t[sl]
        tol = 2e-3 * np.abs(ref) + 1e-3 * np.abs(ref).max() + 1e-30
        assert np.all(np.abs(grad[sl] - ref) <= tol), (kind, grad[sl], ref)
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
    assert l0 == l1 and np.array_equal(np.nan_to_num(g0), np.nan_to_num(g1))
    # the autograd binding returns the same gradient
    F = A.denoise_loss_function()
    theta = torch.tensor(A.params_to_theta(p), dtype=torch.float64, requires_grad=True)
    loss = F.apply(theta, converter, raw, p, target)
    loss.backward()
    assert abs(float(loss.detach()) - l0) <= 1e-6 * l0
    assert np.allclose(theta.grad.numpy()[:30], g0[:30].astype(np.float64), rtol=1e-6, atol=0)
