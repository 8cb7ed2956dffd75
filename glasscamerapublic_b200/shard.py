"""Frame sharding across ranks (one process per GPU).

The raw -> RGB path has no exchange step: frames are independent, so a
batch is split across ranks by pixel count and each rank converts its share
on its own GPU (weak scaling, no data-path collective). The process group
carries the timing reduction (the slowest rank's device time is the job's
time) and, for data-parallel calibration, the one real exchange: the
all-reduce of the per-rank gradient sums (mean_gradient).
"""
from __future__ import annotations


def assign_frames(sizes: list[tuple[int, int]], world: int) -> list[list[int]]:
    """Longest-processing-time assignment of frames (by pixel count) to ranks.

    Deterministic: frames are taken largest first (ties by index) and each
    goes to the least-loaded rank (ties by rank). Returns, per rank, the
    frame indices in ascending order.
    """
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i][0] * sizes[i][1], i))
    load = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += sizes[i][0] * sizes[i][1]
    return [sorted(x) for x in out]


def max_over_ranks(values, dist=None):
    """Element-wise max of a list of floats over all ranks (the job time is
    the slowest rank's). With no process group, returns the values."""
    if dist is None or not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return list(values)
    import torch
    t = torch.tensor(list(values), dtype=torch.float64)
    if dist.get_backend() == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu().tolist()]


def mean_gradient(grad_sum, n_frames: int, dist=None):
    """Data-parallel calibration: the gradient of the mean loss over every
    rank's frames, from this rank's gradient sum over its own frames and its
    frame count. One all-reduce (sum) of len(grad_sum) + 1 FP64 values;
    every rank receives the same vector. With no process group, the local
    mean."""
    import numpy as np
    g = np.asarray(grad_sum, dtype=np.float64)
    if dist is None or not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return g / max(n_frames, 1)
    import torch
    t = torch.tensor(np.append(g, float(n_frames)), dtype=torch.float64)
    if dist.get_backend() == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    t = t.cpu().numpy()
    return t[:-1] / max(t[-1], 1.0)
