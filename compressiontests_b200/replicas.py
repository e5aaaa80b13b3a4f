"""Host logic for running independent units (solves, load cases, meshes, FD probes) on
several GPUs: one process per GPU, units sharded across ranks with no collective on the
data path, timings reduced as the maximum over ranks.  Works with the nccl backend on GPUs
and with gloo on CPU (the tests)."""
from __future__ import annotations

import numpy as np


def shard(n_units, rank, world):
    """Contiguous, balanced range [lo, hi) of n_units for this rank."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(int(n_units), world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def shard_weighted(weights, world):
    """Deterministic longest-processing-time assignment of weighted units (e.g. meshes by
    dof count) to ranks.  Returns a list of unit-index lists, one per rank, each sorted."""
    w = np.asarray(weights, np.float64)
    order = np.lexsort((np.arange(len(w)), -w))   # heaviest first, ties by index
    load = np.zeros(world)
    out = [[] for _ in range(world)]
    for i in order:
        r = int(np.argmin(load))                  # lowest load, lowest rank on ties
        out[r].append(int(i))
        load[r] += w[i]
    return [sorted(o) for o in out]


def max_over_ranks(value, world, device="cpu"):
    """Maximum of a per-rank number over all ranks (the timing rule of multi-GPU runs)."""
    if world == 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_to_root(obj, world, rank):
    """Per-rank Python objects collected on rank 0 (None elsewhere)."""
    if world == 1:
        return [obj]
    import torch.distributed as dist
    out = [None] * world if rank == 0 else None
    dist.gather_object(obj, out, dst=0)
    return out
