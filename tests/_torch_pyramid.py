"""A PyTorch re-expression of the pyramid denoise + reconstruct + output
transform (the oracle's pyramid_denoise, oracle/gls_oracle.hpp, which
restates PyramidProcessor<levels>::denoise, pyramid_processor.cpp:96-172),
in float64 on the CPU, so that torch.autograd gives a reference gradient of
the MSE loss with respect to the per-level parameters. Test infrastructure
only: the product's adjoint is hand-written CUDA (gls_adjoint.cu).

The PCA bases are inputs (held fixed), as in the adjoint. Every function
runs on the device of its inputs; with checkpoint=True the block matching
keeps only one window row's intermediates for the backward pass (it
recomputes them), so a 2048x1536 frame fits on one GPU.
"""
from __future__ import annotations

import math

import torch

ADJ_NPARAMS = 32
LUMA, CHROMA, AY, BY, AC, BC = 0, 5, 10, 15, 20, 25


def theta_from_params(p, levels: int) -> torch.Tensor:
    t = torch.zeros(ADJ_NPARAMS, dtype=torch.float64)
    for l in range(levels):
        t[LUMA + l] = p.denoise[l].luma
        t[CHROMA + l] = p.denoise[l].chroma
        t[AY + l] = p.pyramid_nlf[l].a[0]
        t[BY + l] = p.pyramid_nlf[l].b[0]
        t[AC + l] = p.pyramid_nlf[l].a[1]
        t[BC + l] = p.pyramid_nlf[l].b[1]
    return t


def bilin(img: torch.Tensor, u: torch.Tensor, v: torch.Tensor) -> torch.Tensor:
    """Bilinear sample of img (h, w, C) at texel positions u (w',) x v (h',),
    clamp-to-edge; returns (h', w', C)."""
    h, w = img.shape[:2]
    fu, fv = torch.floor(u), torch.floor(v)
    ax, ay = (u - fu)[None, :, None], (v - fv)[:, None, None]
    x0, y0 = fu.long(), fv.long()
    x0c, x1c = x0.clamp(0, w - 1), (x0 + 1).clamp(0, w - 1)
    y0c, y1c = y0.clamp(0, h - 1), (y0 + 1).clamp(0, h - 1)
    a = img[y0c][:, x0c]
    b = img[y0c][:, x1c]
    c = img[y1c][:, x0c]
    d = img[y1c][:, x1c]
    top = a + (b - a) * ax
    bot = c + (d - c) * ax
    return top + (bot - top) * ay


def downsample(img: torch.Tensor, ow: int, oh: int) -> torch.Tensor:
    h, w = img.shape[:2]
    rx, ry = w / ow, h / oh
    x = torch.arange(ow, dtype=torch.float64, device=img.device)
    y = torch.arange(oh, dtype=torch.float64, device=img.device)
    u0, u1 = x * rx - 0.5, (x + 1) * rx - 0.5
    v0, v1 = y * ry - 0.5, (y + 1) * ry - 0.5
    return 0.25 * (bilin(img, u0, v0) + bilin(img, u1, v0) + bilin(img, u0, v1) + bilin(img, u1, v1))


def smoothstep(e0, e1, x):
    t = torch.clamp((x - e0) / (e1 - e0), 0.0, 1.0)
    return t * t * (3.0 - 2.0 * t)


def subtract_noise(inp, coarse, coarse_den, grad, sharpening, na, nb):
    h, w = inp.shape[:2]
    ch, cw = coarse.shape[:2]
    rx, ry = cw / w, ch / h
    u = (torch.arange(w, dtype=torch.float64, device=inp.device) + 0.5) * rx - 0.5
    v = (torch.arange(h, dtype=torch.float64, device=inp.device) + 0.5) * ry - 0.5
    p1 = bilin(coarse[..., :3], u, v)
    pd = bilin(coarse_den[..., :3], u, v)
    dn = inp[..., :3] - (p1 - pd)  # lumaDenoiseWeight = 1
    if sharpening > 1.0:
        gm = torch.sqrt(grad[..., 0] ** 2 + grad[..., 1] ** 2)
        sigma = torch.sqrt(na + nb * pd[..., 0])
        detail = (smoothstep(sigma, 4 * sigma, gm) * (1 - smoothstep(0.75, 0.95, pd[..., 0])) *
                  smoothstep(0.05, 0.1, pd[..., 0]))
        alpha = (1.0 + (sharpening - 1.0) * detail)[..., None]
    else:
        alpha = torch.full_like(pd[..., :1], sharpening)
    o = pd + (dn - pd) * alpha
    o = torch.cat([torch.clamp(o[..., :1], min=0.0), o[..., 1:]], -1)
    return torch.cat([o, inp[..., 3:4]], -1)


def pca_project(layer, basis):
    h, w = layer.shape[:2]
    lum = layer[..., 0]
    ys = torch.arange(h, device=layer.device)
    xs = torch.arange(w, device=layer.device)
    acc = torch.zeros(h, w, 8, dtype=torch.float64, device=layer.device)
    row = 0
    for j in range(-2, 3):
        for i in range(-2, 3):
            s = lum[(ys + j).clamp(0, h - 1)][:, (xs + i).clamp(0, w - 1)]
            acc = acc + s[..., None] * basis[row][None, None, :]
            row += 1
    return acc


def _window_row(j, layer, pca, L, K1, K2):
    """The five window sums of block_match over the taps of window row j."""
    h, w = layer.shape[:2]
    ys, xs = torch.arange(h, device=layer.device), torch.arange(w, device=layer.device)
    yi = (ys + j).clamp(0, h - 1)
    fy = torch.zeros(h, w, dtype=torch.float64, device=layer.device)
    fcb, fcr, ny, nc = torch.zeros_like(fy), torch.zeros_like(fy), torch.zeros_like(fy), torch.zeros_like(fy)
    for i in range(-10, 11):
        xi = (xs + i).clamp(0, w - 1)
        s = layer[yi][:, xi]
        sp = pca[yi][:, xi]
        d2 = ((sp - pca) ** 2).sum(-1)
        lw = torch.exp(-2.0 * d2 * L * L)
        c1 = (s[..., 1] - layer[..., 1]) * K1
        c2 = (s[..., 2] - layer[..., 2]) * K2
        cw = torch.exp(-2.0 * (lw * lw + c1 * c1 + c2 * c2))
        d = 0.1 * math.sqrt(i * i + j * j)
        sw = math.exp(-2.0 * d * d)
        fy = fy + sw * lw * s[..., 0]
        fcb = fcb + sw * cw * s[..., 1]
        fcr = fcr + sw * cw * s[..., 2]
        ny = ny + sw * lw
        nc = nc + sw * cw
    return fy, fcb, fcr, ny, nc


def block_match(layer, grad, pca, a, b, tm, dp, checkpoint: bool = False):
    """a, b: (3,) tensors of the level's NLF; tm: (luma, chroma, chroma)."""
    y = layer[..., 0]
    dm = [1.0 / (tm[c] * torch.sqrt(a[c] + b[c] * y)) for c in range(3)]
    mag = torch.sqrt(grad[..., 0] ** 2 + grad[..., 1] ** 2)
    sig0 = torch.sqrt(a[0] + b[0] * y)
    edge = smoothstep(2.0, 16.0, dp.gradient_threshold * mag / sig0)
    L = dm[0] / (1.0 + dp.gradient_boost * edge)
    K1, K2 = dm[1] / dp.chroma_boost, dm[2] / dp.chroma_boost
    sums = None
    for j in range(-10, 11):
        if checkpoint:
            from torch.utils.checkpoint import checkpoint as ckpt
            part = ckpt(_window_row, j, layer, pca, L, K1, K2, use_reentrant=False)
        else:
            part = _window_row(j, layer, pca, L, K1, K2)
        sums = part if sums is None else tuple(u + v for u, v in zip(sums, part))
    fy, fcb, fcr, ny, nc = sums
    return torch.stack([fy / ny, fcb / nc, fcr / nc, ny], -1)


def pyramid_rgb(ds, grad, theta, params, bases, y2c, checkpoint: bool = False):
    """Denoised linear camera RGB (h, w, 3) of the despeckled YCbCr image ds
    (h, w, 4) and its gradient (h, w, 2)."""
    L = params.levels
    h, w = ds.shape[:2]
    img = [ds]
    grd = [grad]
    for i in range(1, L):
        img.append(downsample(img[-1][..., :3], w >> i, h >> i))
        img[-1] = torch.cat([img[-1], torch.zeros_like(img[-1][..., :1])], -1)
        grd.append(downsample(grd[-1], w >> i, h >> i))
    den = [None] * L
    for i in range(L - 1, -1, -1):
        dp = params.denoise[i]
        luma, chroma = theta[LUMA + i], theta[CHROMA + i]
        # Cb and Cr NLF tied: one parameter moves both (their calibrated
        # values may differ; the offset between them is held)
        nlf = params.pyramid_nlf[i]
        a = torch.stack([theta[AY + i], theta[AC + i], theta[AC + i] + (float(nlf.a[2]) - float(nlf.a[1]))])
        b = torch.stack([theta[BY + i], theta[BC + i], theta[BC + i] + (float(nlf.b[2]) - float(nlf.b[1]))])
        if i < L - 1:
            layer = subtract_noise(img[i], img[i + 1], den[i + 1], grd[i], dp.sharpening, a[0] * luma, b[0] * luma)
        else:
            layer = img[i]
        pca = pca_project(layer, bases[i])
        den[i] = block_match(layer, grd[i], pca, a, b, (luma, chroma, chroma), dp, checkpoint)
    return den[0][..., :3] @ y2c.T


def loss_and_grad(ds, grad, params, bases, y2c, target, with_ds: bool = False, device: str = "cpu",
                  checkpoint: bool = False):
    """MSE loss and its gradient with respect to the first 30 parameters
    (NaN for the two raw-green entries, which act before ds); with with_ds,
    also dL/d(ds) (h, w, 3). device: where the float64 evaluation runs."""
    f64 = dict(dtype=torch.float64, device=device)
    theta = theta_from_params(params, params.levels).to(device).requires_grad_(True)
    dst = torch.as_tensor(ds, **f64).clone().requires_grad_(with_ds)
    rgb = pyramid_rgb(dst, torch.as_tensor(grad, **f64), theta, params, torch.as_tensor(bases, **f64),
                      torch.as_tensor(y2c, **f64), checkpoint)
    loss = ((rgb - torch.as_tensor(target, **f64)[..., :3]) ** 2).mean()
    loss.backward()
    g = theta.grad.detach().cpu().clone()
    g[30:] = float("nan")
    res = (float(loss.detach()), g.numpy(), rgb.detach().cpu().numpy())
    if with_ds:
        res = res + (dst.grad.detach()[..., :3].cpu().numpy(),)
    return res


def vjp(ds, grad, params, bases, g_out):
    """dL/dtheta (first 30 entries; NaN for the raw-green ones) and dL/d(ds)
    (h, w, 3) of L = sum(g_out * denoised YCbCr), by autograd of the float64
    re-expression (bases held fixed)."""
    theta = theta_from_params(params, params.levels).requires_grad_(True)
    dst = torch.as_tensor(ds, dtype=torch.float64).clone().requires_grad_(True)
    den0 = pyramid_rgb(dst, torch.as_tensor(grad, dtype=torch.float64), theta, params,
                       torch.as_tensor(bases, dtype=torch.float64), torch.eye(3, dtype=torch.float64))
    (den0 * torch.as_tensor(g_out, dtype=torch.float64)[..., :3]).sum().backward()
    g = theta.grad.detach().clone()
    g[30:] = float("nan")
    return g.numpy(), dst.grad.detach()[..., :3].numpy()
