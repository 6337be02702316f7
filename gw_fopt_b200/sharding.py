"""k-hat sharding across ranks (one process per GPU).

Directions are independent units of the spectrum: each k-hat block of the
(K, 2, S, W) output is compute_c_integral on the configuration rotated by
R(k-hat) (rust/bubble-gw/src/many_bubbles/generalized_bulk_flow.rs:928-984 per
rotated frame).  N ranks therefore take disjoint subsets of the directions with
no exchange on the data path: rank r computes directions r, r + N, r + 2N, ...
of a K*N-direction Fibonacci sphere (weak scaling: K directions per rank).  The
only collectives are the timing reduction (max over ranks) and, when a caller
wants the whole spectrum on one rank, one gather of the per-rank blocks.
"""
from __future__ import annotations

import numpy as np

from .workloads import fibonacci_khat

__all__ = ["khat_shard", "max_over_ranks", "gather_spectra"]


def khat_shard(k_per_rank: int, rank: int, world: int) -> np.ndarray:
    """(k_per_rank, 3): this rank's directions of the k_per_rank*world Fibonacci sphere."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    return np.ascontiguousarray(fibonacci_khat(k_per_rank * world)[rank::world])


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over the ranks of the default process group (value itself without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_spectra(local: np.ndarray, rank: int, world: int, dst: int = 0):
    """On rank `dst`: the (K*world, ...) spectrum in Fibonacci-sphere order from every rank's
    (K, ...) block computed on khat_shard(K, rank, world); None on the other ranks."""
    import torch
    import torch.distributed as dist
    if world == 1:
        return local
    arr = np.ascontiguousarray(local)
    cplx = np.iscomplexobj(arr)
    # complex blocks travel as (..., 2) float64 (not every backend moves complex tensors)
    t = torch.from_numpy(arr.view(np.float64).reshape(arr.shape + (2,)) if cplx else arr)
    parts = [torch.empty_like(t) for _ in range(world)] if rank == dst else None
    dist.gather(t, parts, dst=dst)
    if rank != dst:
        return None
    K = local.shape[0]
    full = np.empty((K * world,) + local.shape[1:], dtype=local.dtype)
    for r in range(world):
        p = parts[r].numpy()
        full[r::world] = np.ascontiguousarray(p).view(np.complex128)[..., 0] if cplx else p
    return full
