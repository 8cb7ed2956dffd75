"""The reference gradient for the adjoint checks (CPU, no GPU): the PyTorch
float64 re-expression of the pyramid (tests/_torch_pyramid.py) reproduces
the FP64 oracle's forward, and its autograd gradient agrees with central
finite differences (relative step 1e-3) of the FP64 oracle's loss with the
PCA bases held fixed, to 1e-4 relative."""
import numpy as np
import pytest

import _oracle as O
import _torch_pyramid as TP
from glasscamerapublic_b200 import scene


def _case():
    wl = scene.Workload("adj", 96, 64, levels=3, gain=0.8, read=3.0, iso=400, seed=21)
    raw, clean = scene.make_raw(wl)
    p = scene.make_params(wl)
    st = O.raw_pipeline(raw, p, denoise=True, f64=True, stages=True)
    r = O.pyramid_denoise(st["despeckled"], st["gradient"], p, f64=True)
    _, inv = O.cam_ycbcr(np.eye(3), scene.XYZ_SRGB)
    return wl, p, st["despeckled"], st["gradient"], r, inv, scene.target_rgb(clean)


def _set(p, k, v):
    l, kind = k % 5, k // 5
    if kind == 0:
        p.denoise[l].luma = v
    elif kind == 1:
        p.denoise[l].chroma = v
    elif kind == 2:
        p.pyramid_nlf[l].a[0] = v
    elif kind == 3:
        p.pyramid_nlf[l].b[0] = v
    elif kind == 4:
        d = v - p.pyramid_nlf[l].a[1]
        p.pyramid_nlf[l].a[1] += d
        p.pyramid_nlf[l].a[2] += d
    else:
        d = v - p.pyramid_nlf[l].b[1]
        p.pyramid_nlf[l].b[1] += d
        p.pyramid_nlf[l].b[2] += d


def test_torch_reexpression_matches_oracle_forward():
    wl, p, ds, grad, r, inv, target = _case()
    loss, g, rgb = TP.loss_and_grad(ds, grad, p, r["bases"], inv, target)
    ref = r["out"][..., :3].astype(np.float64) @ np.asarray(inv, np.float64).T
    assert np.abs(rgb - ref).max() < 1e-6  # the oracle's output is stored as float32
    assert abs(loss - O.pyramid_loss(ds, grad, p, r["bases"], inv, target)) < 1e-9 * loss + 1e-15


def test_autograd_matches_oracle_finite_differences():
    wl, p, ds, grad, r, inv, target = _case()
    _, g, _ = TP.loss_and_grad(ds, grad, p, r["bases"], inv, target)
    th = TP.theta_from_params(p, p.levels).numpy()
    checked = 0
    for k in [0, 1, 5, 6, 7, 10, 11, 15, 16, 20, 21, 22, 25, 26, 27]:
        v = th[k]
        h = 1e-3 * abs(v)
        pp, pm = scene.make_params(wl), scene.make_params(wl)
        _set(pp, k, v + h)
        _set(pm, k, v - h)
        lp = O.pyramid_loss(ds, grad, pp, r["bases"], inv, target)
        lm = O.pyramid_loss(ds, grad, pm, r["bases"], inv, target)
        step = TP.theta_from_params(pp, p.levels).numpy()[k] - TP.theta_from_params(pm, p.levels).numpy()[k]
        fd = (lp - lm) / step
        assert abs(fd - g[k]) <= 1e-4 * abs(g[k]) + 1e-12, (k, fd, g[k])
        checked += 1
    assert checked == 15
