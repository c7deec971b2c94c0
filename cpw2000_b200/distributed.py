"""Multi-GPU plumbing: one process per GPU, k-points sharded round-robin.

k-points are independent in H|psi> and in the eigensolver; the only exchange is the
k-weighted reduction of per-k results (forces, stress, band energies) and the
max-over-ranks of timings. ``torch.distributed`` carries both: NCCL on GPUs, gloo on
CPU. No data-path collective: each rank owns whole k-points.
"""
from __future__ import annotations

import numpy as np


def kpoint_shard(nk: int, rank: int, world: int) -> list[int]:
    """The k-points rank `rank` of `world` owns (round-robin)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("invalid rank / world size")
    return list(range(rank, nk, world))


def allreduce_sum(x, device=None) -> np.ndarray:
    """Sum of a float64 array over all ranks (every rank gets the result)."""
    import torch
    import torch.distributed as dist
    t = torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64), device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()


def max_over_ranks(v: float, device=None) -> float:
    """The largest value of `v` over all ranks (device timings of a replicated step)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weighted_kpoint_sum(per_k, weights, nk: int, rank: int, world: int, device=None) -> np.ndarray:
    """sum_k w_k f(k) with each rank evaluating f on its own shard; f(k) -> float64 array."""
    acc = None
    for k in kpoint_shard(nk, rank, world):
        v = weights[k] * np.asarray(per_k(k), dtype=np.float64)
        acc = v if acc is None else acc + v
    if acc is None:
        acc = np.zeros_like(np.asarray(per_k(0), dtype=np.float64))
    return allreduce_sum(acc, device=device)
