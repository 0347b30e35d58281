"""Multi-GPU plumbing: one process per GPU, torch.distributed for rank set-up,
barriers and small result exchanges (NCCL on GPUs, gloo on CPU tests).

The search partitions into independent units, so nothing collective runs on
the data path:
* weak scaling (default): every rank searches its own IF block;
* strong scaling: the PRNs of every signal group are dealt round-robin over
  the ranks, each rank runs its share, and the per-PRN results (bin, offset,
  C/N0, peak, mean, fine Doppler: 32 bytes each) are all-gathered once.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import replace

import numpy as np


def env_ranks() -> tuple[int, int, int]:
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def init(backend: str | None = None, timeout_s: float = 300.0, device=None):
    """Initialises the default process group when WORLD_SIZE > 1; returns
    the torch.distributed module or None for a single process."""
    rank, world, local = env_ranks()
    if world <= 1:
        return None
    import torch
    import torch.distributed as dist
    if not dist.is_initialized():
        be = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        kw = {}
        if be == "nccl" and device is not None:
            kw["device_id"] = device
        dist.init_process_group(be, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return dist


def _tensor(x, dist):
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    return torch.tensor(x, dtype=torch.float64, device=dev)


def max_over_ranks(value: float, dist=None) -> float:
    """The maximum of a per-rank value (device time of the timed region)."""
    if dist is None:
        return float(value)
    t = _tensor([float(value)], dist)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard_groups(groups, rank: int, world: int):
    """The PRNs of each group dealt round-robin over the ranks; returns this
    rank's groups (groups left without PRNs are dropped) and, per kept group,
    the indices of its PRNs in the original group."""
    out, index = [], []
    for gi, g in enumerate(groups):
        sel = list(range(rank, len(g.prns), world))
        if not sel:
            continue
        out.append(replace(g, prns=[g.prns[i] for i in sel]))
        index.append((gi, sel))
    return out, index


def gather_results(local: np.ndarray, index, groups, world: int, dist=None) -> list:
    """All-gathers per-PRN result records (numpy structured array in the
    order of this rank's sharded groups) and returns, on every rank, one array
    per original group in PRN order."""
    if dist is None:
        parts = [(local, index)]
    else:
        parts = [None] * world
        dist.all_gather_object(parts, (local, index))
    out = [np.zeros(len(g.prns), local.dtype) for g in groups]
    for arr, idx in parts:
        k = 0
        for gi, sel in idx:
            out[gi][sel] = arr[k:k + len(sel)]
            k += len(sel)
    return out
