"""Frame sharding across ranks (one process per GPU).

The raw -> RGB path has no exchange step: frames are independent, so a
batch is split across ranks by pixel count and each rank converts its share
on its own GPU (weak scaling, no data-path collective). The process group
carries the timing reduction (the slowest rank's device time is the job's
time) and, for data-parallel calibration, the one real exchange: the
all-reduce of the per-rank gradient sums (mean_gradient).

A burst splits by member (burst_members): rank 0 detects the reference
frame and broadcasts its features (broadcast_features), every rank
registers and warps its own members, the homographies are all-gathered
(all_gather_rows) and the per-rank running means are reduced to rank 0
(reduce_mean). Collective tensors live on the GPU under NCCL and on the
host under gloo.
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


def burst_members(n_frames: int, world: int) -> list[list[int]]:
    """Burst members per rank: member m (0 the reference frame) goes to
    rank m % world, so rank 0 holds the reference frame, whose features it
    detects and broadcasts, and every rank registers and warps its own
    members against them."""
    if world < 1:
        raise ValueError("world must be >= 1")
    if n_frames < 1:
        raise ValueError("a burst has at least one frame")
    return [list(range(r, n_frames, world)) for r in range(world)]


def _comm_device(dist, like=None):
    """Where a collective's tensors live: CUDA for NCCL, host for gloo."""
    import torch
    if dist.get_backend() == "nccl":
        return like.device if like is not None and like.is_cuda else torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def _active(dist) -> bool:
    return dist is not None and dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1


def broadcast_bytes(payload: bytes | None, dist=None, src: int = 0) -> bytes:
    """Broadcast of a byte string of any length from src (two collectives:
    the length, then the bytes). Every rank receives src's bytes."""
    if not _active(dist):
        return bytes(payload)
    import torch
    dev = _comm_device(dist)
    n = torch.tensor([len(payload) if dist.get_rank() == src else 0], dtype=torch.int64, device=dev)
    dist.broadcast(n, src)
    buf = torch.zeros(int(n.item()), dtype=torch.uint8, device=dev)
    if dist.get_rank() == src and len(payload):
        buf.copy_(torch.frombuffer(bytearray(payload), dtype=torch.uint8))
    if buf.numel():
        dist.broadcast(buf, src)
    return bytes(buf.cpu().numpy().tobytes())


def broadcast_features(kps, desc, dist=None, src: int = 0):
    """The reference frame's keypoints (28-byte records) and descriptors
    ([n][64] float32) from src to every rank: the count, then the records,
    then the descriptors (three collectives, about 0.4 MB at 1500 features).
    Returns torch tensors (keypoint bytes as uint8 [n * 28], descriptors
    float32 [n][64]) on the collective's device: CUDA under NCCL, so that
    they load into a detector slot without a host round trip."""
    import numpy as np
    import torch
    if not _active(dist):
        k = torch.from_numpy(np.ascontiguousarray(kps).view(np.uint8).reshape(-1).copy())
        return k, torch.from_numpy(np.ascontiguousarray(desc, np.float32).reshape(-1, 64).copy())
    from . import KEYPOINT_DTYPE
    dev = _comm_device(dist)
    me = dist.get_rank() == src
    rec = KEYPOINT_DTYPE.itemsize
    n = torch.tensor([len(kps) if me else 0], dtype=torch.int64, device=dev)
    dist.broadcast(n, src)
    n = int(n.item())
    kb = torch.zeros(n * rec, dtype=torch.uint8, device=dev)
    db = torch.zeros((n, 64), dtype=torch.float32, device=dev)
    if me and n:
        kb.copy_(torch.from_numpy(np.ascontiguousarray(kps).view(np.uint8).reshape(-1).copy()))
        db.copy_(torch.from_numpy(np.ascontiguousarray(desc, np.float32).reshape(n, 64)))
    if n:
        dist.broadcast(kb, src)
        dist.broadcast(db, src)
    return kb, db


def all_gather_rows(rows, mine: list[int], n: int, dist=None):
    """Rows of an [n][k] float32 array that ranks hold disjoint parts of
    (this rank the rows `mine`): every rank receives the whole array (one
    all-reduce of the zero-filled array; each row has one nonzero source,
    so the sum is exact)."""
    import numpy as np
    a = np.asarray(rows, np.float32)
    out = np.zeros((n,) + a.shape[1:], np.float32)
    if len(mine):
        out[mine] = a
    if not _active(dist):
        return out
    import torch
    t = torch.from_numpy(out).to(_comm_device(dist))
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()


def reduce_mean(partial_mean, count: int, total: int, dist=None, dst: int = 0):
    """The mean over all ranks' frames from each rank's running mean of its
    own `count` frames (partial_mean, a float32 tensor; ignored when count
    is 0): one reduce (sum) of count * partial_mean to dst, divided by
    `total` there. Returns the mean on dst (on partial_mean's device) and
    None elsewhere."""
    import torch
    if not _active(dist):
        return partial_mean
    dev = _comm_device(dist, partial_mean)
    t = (partial_mean.to(dev) * float(count)) if count > 0 else torch.zeros_like(partial_mean, device=dev)
    dist.reduce(t, dst, op=dist.ReduceOp.SUM)
    if dist.get_rank() != dst:
        return None
    return (t / float(total)).to(partial_mean.device)
