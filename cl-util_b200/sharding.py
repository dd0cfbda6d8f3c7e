"""Work split and timing across ranks (one process per GPU).

Grids are independent units, so several GPUs share a batch by giving each rank whole grids:
``lpt_assign`` is the longest-processing-time greedy rule on pixel count (largest grid first,
to the least-loaded rank), which keeps the slowest rank within 4/3 of the best split.  There
is no collective on the solve path; only the per-rank timings and checks are reduced, with
``reduce_max`` / ``reduce_min`` (NCCL on GPUs, gloo on the CPU).
"""
from __future__ import annotations


def lpt_assign(weights, n: int):
    """Indices of `weights` for each of `n` ranks: largest weight first, each to the rank with
    the smallest load so far (ties: lower index, lower rank).  Deterministic, so every rank
    computes the same split without communicating."""
    if n < 1:
        raise ValueError("n must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    loads = [0] * n
    out = [[] for _ in range(n)]
    for i in order:
        k = min(range(n), key=lambda r: (loads[r], r))
        out[k].append(i)
        loads[k] += weights[i]
    for lst in out:
        lst.sort()
    return out


def _reduce(value: float, op, device):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def reduce_max(value: float, device="cpu") -> float:
    """Largest value over all ranks (a job's time is its slowest rank's)."""
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.MAX, device)


def reduce_min(value: float, device="cpu") -> float:
    """Smallest value over all ranks (a check passes only when it passes everywhere)."""
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.MIN, device)


def reduce_sum(value: float, device="cpu") -> float:
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.SUM, device)
