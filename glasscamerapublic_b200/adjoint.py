"""Differentiable calibration: the hand-written adjoint of the FP32 raw path
(gls_demosaic_denoise_vjp) behind a thin torch.autograd.Function, so that
the 32 calibration scalars can be tuned by gradient descent and checked
against finite differences and a reference autograd gradient.

Parameter vector layout (GLS_ADJ_*): luma[5], chroma[5], A_Y[5], B_Y[5],
A_C[5], B_C[5] of the pyramid levels, then the raw green a and b (the
means of raw_nlf a[1], a[3] and of b[1], b[3], which move together).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import (ADJ_NLF_AC, ADJ_NLF_AY, ADJ_NLF_BC, ADJ_NLF_BY, ADJ_CHROMA, ADJ_LUMA, ADJ_NPARAMS, F32, HOST_IO,
               DemosaicParams, ImageView, check, lib)
from .api import _ptr, _row_stride, _stream_handle


def params_to_theta(p: DemosaicParams) -> np.ndarray:
    t = np.zeros(ADJ_NPARAMS, np.float64)
    for l in range(p.levels):
        t[ADJ_LUMA + l] = p.denoise[l].luma
        t[ADJ_CHROMA + l] = p.denoise[l].chroma
        t[ADJ_NLF_AY + l] = p.pyramid_nlf[l].a[0]
        t[ADJ_NLF_BY + l] = p.pyramid_nlf[l].b[0]
        t[ADJ_NLF_AC + l] = p.pyramid_nlf[l].a[1]
        t[ADJ_NLF_BC + l] = p.pyramid_nlf[l].b[1]
    t[30] = (p.raw_nlf.a[1] + p.raw_nlf.a[3]) / 2
    t[31] = (p.raw_nlf.b[1] + p.raw_nlf.b[3]) / 2
    return t


def theta_to_params(theta, base: DemosaicParams) -> DemosaicParams:
    """A copy of base with the parameters set from theta. Cb and Cr NLF move
    together, keeping their calibrated offset; so do the raw G and G2
    variance coefficients."""
    p = DemosaicParams.from_buffer_copy(base)
    th = np.asarray(theta, np.float64)
    for l in range(base.levels):
        p.denoise[l].luma = th[ADJ_LUMA + l]
        p.denoise[l].chroma = th[ADJ_CHROMA + l]
        p.pyramid_nlf[l].a[0] = th[ADJ_NLF_AY + l]
        p.pyramid_nlf[l].b[0] = th[ADJ_NLF_BY + l]
        da = th[ADJ_NLF_AC + l] - base.pyramid_nlf[l].a[1]
        db = th[ADJ_NLF_BC + l] - base.pyramid_nlf[l].b[1]
        p.pyramid_nlf[l].a[1] = base.pyramid_nlf[l].a[1] + da
        p.pyramid_nlf[l].a[2] = base.pyramid_nlf[l].a[2] + da
        p.pyramid_nlf[l].b[1] = base.pyramid_nlf[l].b[1] + db
        p.pyramid_nlf[l].b[2] = base.pyramid_nlf[l].b[2] + db
    t0 = params_to_theta(base)
    for k, arr in ((30, "a"), (31, "b")):
        d = th[k] - t0[k]
        for c in (1, 3):
            getattr(p.raw_nlf, arr)[c] = getattr(base.raw_nlf, arr)[c] + d
    return p


def loss_and_grad(converter, raw, params: DemosaicParams, target, stream=None):
    """(MSE loss, dL/dtheta [32]) of the FP32 raw -> RGB path for one frame.
    raw: uint16 (h, w) numpy array or CUDA tensor; target: float32 (h, w, 3|4)
    of the same kind."""
    h, w = raw.shape
    host = isinstance(raw, np.ndarray)
    if host:
        raw = np.ascontiguousarray(raw, np.uint16)
        target = np.ascontiguousarray(target, np.float32)
    tv = ImageView(C.c_void_p(_ptr(target)), w, h, target.shape[2], F32, _row_stride(target))
    loss = C.c_double(0)
    grad = np.zeros(ADJ_NPARAMS, np.float32)
    check(lib().gls_demosaic_denoise_vjp(converter.handle, C.c_void_p(_ptr(raw)), w, h, _row_stride(raw),
                                         C.byref(params), C.byref(tv), HOST_IO if host else 0, C.byref(loss),
                                         grad.ctypes.data_as(C.POINTER(C.c_float)), _stream_handle(stream)))
    return loss.value, grad


def denoise_loss_function():
    """torch.autograd.Function: loss = f(theta) over one frame, the gradient
    from the hand-written adjoint."""
    import torch

    class DenoiseLoss(torch.autograd.Function):
        @staticmethod
        def forward(ctx, theta, converter, raw, base_params, target):
            p = theta_to_params(theta.detach().cpu().numpy(), base_params)
            loss, g = loss_and_grad(converter, raw, p, target)
            gt = torch.from_numpy(g.astype(np.float64)).to(theta.dtype)
            ctx.save_for_backward(gt)
            return theta.new_tensor(loss)

        @staticmethod
        def backward(ctx, gout):
            (gt,) = ctx.saved_tensors
            return gt.to(gout.device) * gout, None, None, None, None

    return DenoiseLoss
