"""Pyramid burst fusion (gls_fuse_pyramid) on the GPU.

  * uniform weights reduce to the flat mean of the warped frames, i.e. the
    output of the reference's registerAndFuse running mean (1e-5);
  * against a float64 numpy restatement of the Laplacian fusion (warp with
    the library's registerImage, which is bit-exact to the oracle; the
    oracle's down-sampling; bilinear up-sampling), 1e-4;
  * robust weights keep an outlier frame's content out of the result.
"""
import numpy as np
import pytest
import torch

import _oracle as O
from glasscamerapublic_b200 import scene
from glasscamerapublic_b200.registration import SURF, RegisterAndFuseKernel, fuse_pyramid, register_image

pytestmark = pytest.mark.gpu


def _frames(n=4, w=160, h=120, seed=0):
    rng = np.random.default_rng(seed)
    base = scene.textured_scene(w, h, seed)
    frames, Hs = [np.concatenate([base, np.zeros((h, w, 1), np.float32)], -1)], [np.eye(3, dtype=np.float32)]
    for f in range(1, n):
        H = np.array([[1, 0.002 * f, 1.5 * f], [-0.003 * f, 1, -0.75 * f], [0, 0, 1]], np.float32)
        noisy = base + rng.normal(0, 0.02, base.shape).astype(np.float32)
        frames.append(np.concatenate([noisy, np.zeros((h, w, 1), np.float32)], -1))
        Hs.append(H)
    return frames, Hs


def _warped(frames, Hs):
    out = []
    for f, H in zip(frames, Hs):
        t = torch.from_numpy(f).cuda()
        o = torch.empty_like(t)
        register_image(t, o, H)
        out.append(o.cpu().numpy().astype(np.float64))
    return out


def _up(c, w, h):
    ch, cw = c.shape[:2]
    u = (np.arange(w) + 0.5) * np.float32(cw / w) - 0.5
    v = (np.arange(h) + 0.5) * np.float32(ch / h) - 0.5
    x0, y0 = np.floor(u).astype(int), np.floor(v).astype(int)
    ax, ay = (u - x0)[None, :, None], (v - y0)[:, None, None]
    X0, X1 = np.clip(x0, 0, cw - 1), np.clip(x0 + 1, 0, cw - 1)
    Y0, Y1 = np.clip(y0, 0, ch - 1), np.clip(y0 + 1, 0, ch - 1)
    a, b, cc, d = c[Y0][:, X0], c[Y0][:, X1], c[Y1][:, X0], c[Y1][:, X1]
    top, bot = a + (b - a) * ax, cc + (d - cc) * ax
    return top + (bot - top) * ay


def _numpy_fusion(warped, levels, robustness):
    h, w = warped[0].shape[:2]
    pyrs = []
    for img in warped:
        g = [img[..., :3]]
        for l in range(1, levels):
            rgba = np.concatenate([g[-1], np.zeros(g[-1].shape[:2] + (1,))], -1).astype(np.float32)
            g.append(O.downsample(rgba, w >> l, h >> l, f64=True)[..., :3].astype(np.float64))
        bands = [g[l] - _up(g[l + 1], w >> l, h >> l) for l in range(levels - 1)] + [g[-1]]
        pyrs.append(bands)
    fused = []
    for l in range(levels):
        num = pyrs[0][l].copy()
        den = np.ones(num.shape[:2] + (1,))
        for p in pyrs[1:]:
            wgt = np.exp(-robustness * ((p[l] - pyrs[0][l]) ** 2).sum(-1, keepdims=True)) if robustness > 0 else 1.0
            num += wgt * p[l]
            den += wgt
        fused.append(num / den)
    out = fused[-1]
    for l in range(levels - 2, -1, -1):
        out = fused[l] + _up(out, w >> l, h >> l)
    return out


@pytest.fixture(scope="module")
def ctx():
    s = SURF(64, 64, max_features=10)
    yield s
    s.close()


@pytest.mark.parametrize("levels", [1, 3, 5])
def test_uniform_fusion_is_the_flat_mean(ctx, levels):
    frames, Hs = _frames()
    warped = _warped(frames, Hs)
    mean = np.mean([w[..., :3] for w in warped], 0)
    t = [torch.from_numpy(f).cuda() for f in frames]
    out = torch.empty_like(t[0])
    fuse_pyramid(ctx, t, Hs, out, levels=levels, robustness=0.0)
    torch.cuda.synchronize()
    got = out.cpu().numpy()[..., :3]
    assert np.abs(got - mean).max() < 1e-5
    # registerAndFuse's running mean (count f + 1)
    run = t[0].clone()
    for f in range(1, len(t)):
        RegisterAndFuseKernel()(run, t[f], run, Hs[f], f + 1)
    torch.cuda.synchronize()
    assert np.abs(run.cpu().numpy()[..., :3] - got).max() < 1e-5


@pytest.mark.parametrize("robustness", [0.0, 50.0, 400.0])
def test_fusion_matches_numpy_restatement(ctx, robustness):
    frames, Hs = _frames(seed=1)
    warped = _warped(frames, Hs)
    ref = _numpy_fusion(warped, 4, robustness)
    t = [torch.from_numpy(f).cuda() for f in frames]
    out = torch.empty_like(t[0])
    fuse_pyramid(ctx, t, Hs, out, levels=4, robustness=robustness)
    torch.cuda.synchronize()
    assert np.abs(out.cpu().numpy()[..., :3] - ref).max() < 1e-4


def test_robust_weights_reject_an_outlier_frame(ctx):
    frames, _ = _frames(n=4, seed=2)
    Hs = [np.eye(3, dtype=np.float32)] * 4
    bad = frames[2].copy()
    bad[40:80, 50:100, :3] = 1.0  # an object that moved in one frame
    frames[2] = bad
    t = [torch.from_numpy(f).cuda() for f in frames]
    flat, robust = torch.empty_like(t[0]), torch.empty_like(t[0])
    fuse_pyramid(ctx, t, Hs, flat, levels=4, robustness=0.0)
    fuse_pyramid(ctx, t, Hs, robust, levels=4, robustness=200.0)
    torch.cuda.synchronize()
    region = (slice(45, 75), slice(55, 95), slice(0, 3))
    e_flat = np.abs(flat.cpu().numpy()[region] - frames[0][region]).mean()
    e_rob = np.abs(robust.cpu().numpy()[region] - frames[0][region]).mean()
    assert e_rob < 0.2 * e_flat, (e_rob, e_flat)
