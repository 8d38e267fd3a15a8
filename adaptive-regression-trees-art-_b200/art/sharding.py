"""Multi-GPU plumbing for the batched path: one process per GPU, no data-path collective.

Every unit of the hot path is independent (ridge systems, split nodes, chains,
surrogate jobs), so N GPUs run N shards side by side.  Two layouts:

* weak scaling -- each rank generates and solves its own batch (``rank_seed``);
* strong scaling -- one batch is cut into contiguous segment ranges whose
  costs ``sum n * (p + 1)^2`` are balanced (``balanced_shards``), the
  partition the reference's batched workspaces would need to span devices.

The only collective is the timing reduction: device times are combined as the
maximum over ranks (``max_over_ranks``), on NCCL for CUDA tensors and on gloo
for CPU tensors, with every rank taking the same steps in the same order.
"""

from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

__all__ = ["RankInfo", "rank_info", "rank_seed", "balanced_shards", "max_over_ranks", "sum_over_ranks"]


@dataclass(frozen=True)
class RankInfo:
    rank: int
    world: int
    local: int


def rank_info() -> RankInfo:
    """Rank, world size and local rank from the launcher's environment (torchrun)."""

    return RankInfo(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
                    int(os.environ.get("LOCAL_RANK", "0")))


def rank_seed(base: int, rank: int) -> int:
    """Seed of rank ``rank``'s own batch under weak scaling."""

    return int(base) + int(rank)


def balanced_shards(row_counts, feature_counts, world: int) -> np.ndarray:
    """Contiguous segment boundaries [world + 1] with near-equal solve cost.

    Cost of segment k is ``n_k * (p_k + 1)^2`` (Gram formation dominates).
    Boundary r is the first segment whose cost prefix reaches r/world of the
    total, so shards are contiguous, cover every segment exactly once and
    differ from the ideal share by at most one segment's cost.
    """

    if world < 1:
        raise ValueError("world must be at least 1")
    n = np.asarray(row_counts, dtype=np.float64).reshape(-1)
    p = np.asarray(feature_counts, dtype=np.float64).reshape(-1)
    if n.shape != p.shape:
        raise ValueError("row_counts and feature_counts must have the same length")
    if np.any(n < 0) or np.any(p < 1):
        raise ValueError("row counts must be >= 0 and feature counts >= 1")
    K = n.size
    cost = n * (p + 1.0) ** 2
    prefix = np.concatenate([[0.0], np.cumsum(cost)])
    total = prefix[-1]
    bounds = np.empty(world + 1, dtype=np.int64)
    bounds[0], bounds[-1] = 0, K
    for r in range(1, world):
        if total <= 0.0:
            bounds[r] = (K * r) // world
        else:
            bounds[r] = int(np.searchsorted(prefix, total * r / world, side="left"))
        bounds[r] = min(max(bounds[r], bounds[r - 1]), K)
    return bounds


def _reduce(value: float, op_name: str, device=None) -> float:
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op_name))
    return float(t.item())


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank scalar (device time of the timed region) over all ranks."""

    return _reduce(value, "MAX", device)


def sum_over_ranks(value: float, device=None) -> float:
    """Sum of a per-rank scalar (units processed) over all ranks."""

    return _reduce(value, "SUM", device)
