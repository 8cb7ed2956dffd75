"""Calibration tuning by gradient descent: the per-level denoise strengths
and noise-model coefficients of a CameraCalibration
(CameraCalibration.hpp:24-39, iPhone14WideCalibration.cpp:151-252 for the
tables it starts from) fitted to frames with known clean targets, through
the hand-written adjoint (gls_demosaic_denoise_vjp).

The optimiser is Adam (Kingma & Ba, 2015) with a per-parameter step scale:
each scalar moves by lr x its starting magnitude x the normalised Adam
direction, because the 32 scalars span many decades (NLF coefficients near
1e-5, strengths near 1). Every step is projected onto the box the
parameters live in (strengths and NLF slopes positive). Data-parallel
tuning averages the ranks' gradients with one all-reduce per step
(shard.mean_gradient); every rank then takes the same step.

State (parameters, Adam moments, step count, loss history) is written to
and read from JSON, so a run can stop and resume bit for bit.
"""
from __future__ import annotations

import json
import math
from pathlib import Path
from typing import Callable, Sequence

import numpy as np

from . import ADJ_CHROMA, ADJ_LUMA, ADJ_NLF_AC, ADJ_NLF_AY, ADJ_NLF_BC, ADJ_NLF_BY, ADJ_NPARAMS

# lower bounds of the box: strengths and variance slopes stay positive; the
# NLF intercepts may go negative (a fitted noise floor can be below zero)
# but not below minus their starting magnitude
_POSITIVE = ([ADJ_LUMA + l for l in range(5)] + [ADJ_CHROMA + l for l in range(5)] +
             [ADJ_NLF_BY + l for l in range(5)] + [ADJ_NLF_BC + l for l in range(5)] + [31])
_INTERCEPTS = [ADJ_NLF_AY + l for l in range(5)] + [ADJ_NLF_AC + l for l in range(5)] + [30]


class AdamBox:
    """Adam on a parameter vector with per-parameter step scales and a box
    projection. Plain numpy, FP64; deterministic."""

    def __init__(self, theta0, scale, lo, hi, lr: float = 0.05, betas=(0.9, 0.999), eps: float = 1e-8):
        self.theta = np.array(theta0, np.float64)
        self.scale = np.array(scale, np.float64)
        self.lo = np.array(lo, np.float64)
        self.hi = np.array(hi, np.float64)
        self.lr, self.b1, self.b2, self.eps = float(lr), float(betas[0]), float(betas[1]), float(eps)
        self.m = np.zeros_like(self.theta)
        self.v = np.zeros_like(self.theta)
        self.t = 0

    def step(self, grad) -> np.ndarray:
        g = np.asarray(grad, np.float64) * self.scale  # the gradient in scaled coordinates
        self.t += 1
        self.m = self.b1 * self.m + (1.0 - self.b1) * g
        self.v = self.b2 * self.v + (1.0 - self.b2) * g * g
        mh = self.m / (1.0 - self.b1 ** self.t)
        vh = self.v / (1.0 - self.b2 ** self.t)
        self.theta = np.clip(self.theta - self.lr * self.scale * mh / (np.sqrt(vh) + self.eps), self.lo, self.hi)
        return self.theta

    def state(self) -> dict:
        return {"theta": self.theta.tolist(), "scale": self.scale.tolist(), "lo": self.lo.tolist(),
                "hi": self.hi.tolist(), "lr": self.lr, "betas": [self.b1, self.b2], "eps": self.eps,
                "m": self.m.tolist(), "v": self.v.tolist(), "t": self.t}

    @classmethod
    def from_state(cls, s: dict) -> "AdamBox":
        o = cls(s["theta"], s["scale"], s["lo"], s["hi"], s["lr"], tuple(s["betas"]), s["eps"])
        o.m = np.array(s["m"], np.float64)
        o.v = np.array(s["v"], np.float64)
        o.t = int(s["t"])
        return o


def default_box(theta0):
    """Step scales and bounds for a starting parameter vector. Entries that
    start at zero (the levels a pyramid does not have) stay frozen."""
    t0 = np.asarray(theta0, np.float64)
    mag = np.abs(t0)
    lo = np.full(ADJ_NPARAMS, -np.inf)
    hi = np.full(ADJ_NPARAMS, np.inf)
    for k in _POSITIVE:
        lo[k] = 1e-3 * mag[k]
    for k in _INTERCEPTS:
        lo[k] = -mag[k]
    frozen = mag == 0
    lo[frozen] = hi[frozen] = t0[frozen]
    return mag, lo, hi


GradFn = Callable[[np.ndarray, int], "tuple[float, np.ndarray]"]


class CalibrationTuner:
    """Fits the 32 calibration scalars (layout GLS_ADJ_*) to frames with
    clean targets.

    grad_fn(theta, i) -> (loss_i, dL_i/dtheta) for this rank's frame i; the
    default, built by for_frames(), runs the FP32 raw path forward and its
    adjoint on the GPU. Each step sums the loss and gradient over this
    rank's frames, averages both over every rank's frames (one all-reduce
    when dist holds a process group), and takes one Adam step; every rank
    ends the step with the same parameters.
    """

    def __init__(self, theta0, grad_fn: GradFn, n_frames: int, lr: float = 0.05, dist=None,
                 scale=None, lo=None, hi=None):
        if n_frames < 0:
            raise ValueError("n_frames must be >= 0")
        s, l, h = default_box(theta0)
        self.opt = AdamBox(theta0, s if scale is None else scale, l if lo is None else lo,
                           h if hi is None else hi, lr)
        self.grad_fn = grad_fn
        self.n_frames = int(n_frames)
        self.dist = dist
        self.history: list[float] = []

    @property
    def theta(self) -> np.ndarray:
        return self.opt.theta.copy()

    def evaluate(self, theta=None) -> "tuple[float, np.ndarray]":
        """Mean loss and gradient over every rank's frames at theta."""
        from .shard import mean_gradient
        th = self.opt.theta if theta is None else np.asarray(theta, np.float64)
        acc = np.zeros(ADJ_NPARAMS + 1, np.float64)
        for i in range(self.n_frames):
            loss, g = self.grad_fn(th, i)
            acc[:ADJ_NPARAMS] += np.asarray(g, np.float64)
            acc[ADJ_NPARAMS] += float(loss)
        m = mean_gradient(acc, self.n_frames, self.dist)
        return float(m[ADJ_NPARAMS]), m[:ADJ_NPARAMS]

    def step(self) -> float:
        """One Adam step; returns the mean loss at the parameters the step
        started from."""
        loss, g = self.evaluate()
        if not (math.isfinite(loss) and np.all(np.isfinite(g))):
            raise FloatingPointError(f"non-finite loss or gradient at step {self.opt.t}")
        self.opt.step(g)
        self.history.append(loss)
        return loss

    def run(self, steps: int, checkpoint: "str | Path | None" = None, every: int = 1) -> list[float]:
        """steps Adam steps; with checkpoint, the state is written there
        every `every` steps and after the last (by rank 0 alone under a
        process group)."""
        out = []
        for k in range(steps):
            out.append(self.step())
            if checkpoint is not None and ((k + 1) % max(every, 1) == 0 or k + 1 == steps):
                self.save(checkpoint)
        return out

    # -- checkpoint / resume ------------------------------------------------

    def state_dict(self) -> dict:
        return {"format": "glscam-calibration-tuner", "version": 1, "n_params": ADJ_NPARAMS,
                "adam": self.opt.state(), "history": list(self.history)}

    def load_state_dict(self, s: dict) -> None:
        if s.get("format") != "glscam-calibration-tuner" or s.get("n_params") != ADJ_NPARAMS:
            raise ValueError("not a calibration tuner state")
        self.opt = AdamBox.from_state(s["adam"])
        self.history = [float(v) for v in s["history"]]

    def save(self, path) -> None:
        if self.dist is not None and self.dist.is_available() and self.dist.is_initialized() \
                and self.dist.get_rank() != 0:
            return
        p = Path(path)
        tmp = p.with_name(p.name + ".tmp")
        tmp.write_text(json.dumps(self.state_dict()))
        tmp.replace(p)  # a reader never sees a half-written file

    def load(self, path) -> None:
        self.load_state_dict(json.loads(Path(path).read_text()))

    # -- GPU frames ---------------------------------------------------------

    @classmethod
    def for_frames(cls, converter, frames: Sequence, targets: Sequence, base_params, lr: float = 0.05,
                   dist=None, stream=None) -> "CalibrationTuner":
        """A tuner over this rank's frames (uint16 raw arrays or CUDA
        tensors) and their float32 targets, starting from base_params: each
        loss and gradient comes from gls_demosaic_denoise_vjp."""
        from .adjoint import loss_and_grad, params_to_theta, theta_to_params
        if len(frames) != len(targets):
            raise ValueError("frames and targets differ in length")

        def grad_fn(theta, i):
            return loss_and_grad(converter, frames[i], theta_to_params(theta, base_params), targets[i], stream)

        t = cls(params_to_theta(base_params), grad_fn, len(frames), lr, dist)
        t.base_params = base_params
        return t

    @staticmethod
    def job_share(sizes, dist=None) -> list[int]:
        """This rank's frames of a job of frames with the given (width,
        height): the pixel-count split of shard.assign_frames, all frames
        without a process group."""
        from .shard import assign_frames
        active = dist is not None and dist.is_available() and dist.is_initialized()
        world, rank = (dist.get_world_size(), dist.get_rank()) if active else (1, 0)
        return assign_frames([(int(w), int(h)) for w, h in sizes], world)[rank]

    @classmethod
    def for_job(cls, converter, frames: Sequence, targets: Sequence, base_params, lr: float = 0.05,
                dist=None, stream=None) -> "CalibrationTuner":
        """for_frames over this rank's share of the whole job's frames
        (job_share of their sizes). Every rank passes the same lists; each
        steps on the mean over all of them."""
        if len(frames) != len(targets):
            raise ValueError("frames and targets differ in length")
        mine = cls.job_share([(f.shape[1], f.shape[0]) for f in frames], dist)
        return cls.for_frames(converter, [frames[i] for i in mine], [targets[i] for i in mine], base_params, lr,
                              dist, stream)

    def params(self):
        """The current parameters as DemosaicParams (tuners from for_frames)."""
        from .adjoint import theta_to_params
        return theta_to_params(self.opt.theta, self.base_params)
