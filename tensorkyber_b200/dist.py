"""Multi-process plumbing for running the transforms on several GPUs.

The path partitions trivially: polynomials (and matrix-vector jobs) are
independent, so N processes (one per GPU) each transform a contiguous range
of the batch and there is no exchange step on the data path.  This module
holds the host-side pieces: reading the launcher's environment, the
contiguous shard of each rank, the max-over-ranks timing reduction, and
gathering shards back to one rank.  They run on NCCL between GPUs (the
buffers they exchange then live on the rank's current CUDA device) and on
gloo on the CPU (tests).
"""
from __future__ import annotations

import datetime
import os

import numpy as np


def env():
    """(rank, world_size, local_rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, timeout_s: float = 120.0, device=None):
    """Initialise the default process group when WORLD_SIZE > 1; returns the
    torch.distributed module, or None for a single process."""
    rank, world, _ = env()
    if world <= 1:
        return None
    import torch.distributed as dist
    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if device is not None:
        kw["device_id"] = device
    dist.init_process_group(backend, **kw)
    return dist


def shard(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous range [start, stop) of n items owned by `rank`: ranks differ
    by at most one item and the ranges tile [0, n) in rank order."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError("bad shard request")
    return rank * n // world, (rank + 1) * n // world


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The maximum of a per-rank scalar (elapsed time) over all ranks."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_shards(local: np.ndarray, n: int, dist=None, dst: int = 0, device=None):
    """Concatenates every rank's shard (rank order) on rank `dst`; returns the
    full (n, ...) array there and None elsewhere.  Shards follow shard().
    Point-to-point buffers go on `device`: by default the current CUDA device
    under NCCL (which moves only CUDA tensors) and host memory otherwise."""
    if dist is None:
        return local
    import torch
    if device is None:
        device = (torch.device("cuda", torch.cuda.current_device())
                  if dist.get_backend() == "nccl" else torch.device("cpu"))
    rank, world = dist.get_rank(), dist.get_world_size()
    start, stop = shard(n, rank, world)
    if local.shape[0] != stop - start:
        raise ValueError("local shard does not match shard()")
    tail = local.shape[1:]
    if rank == dst:
        out = np.empty((n,) + tail, dtype=local.dtype)
        out[start:stop] = local
        for r in range(world):
            if r == dst:
                continue
            a, b = shard(n, r, world)
            buf = torch.empty((b - a,) + tail, dtype=torch.from_numpy(local[:0]).dtype,
                              device=device)
            dist.recv(buf, src=r)
            out[a:b] = buf.cpu().numpy()
        return out
    dist.send(torch.from_numpy(np.ascontiguousarray(local)).to(device), dst=dst)
    return None
