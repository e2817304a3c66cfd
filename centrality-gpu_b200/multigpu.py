"""Multi-GPU plumbing for the BC engine: one process per GPU.

The work units of a plan (independent source passes) are dealt round-robin
to the ranks — no data-path collective while they run (weak scaling); each
rank's BC contributions are then combined by one FP64 all-reduce over NCCL
(gloo on CPU). Every rank takes the same collective steps in the same order.
"""
from __future__ import annotations

import numpy as np


def shard(items, rank: int, world: int):
    """The items rank `rank` of `world` processes (round-robin)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    return list(items)[rank::world]


def combine_bc(local_contrib, art, dist=None, device=None):
    """Sums per-rank BC contributions (without articulation terms) over all
    ranks and adds the articulation terms once. Returns a numpy FP64 array."""
    local = np.asarray(local_contrib, dtype=np.float64)
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return local + np.asarray(art, dtype=np.float64)
    import torch
    t = torch.from_numpy(local.copy())
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t)  # FP64 sum over ranks
    return t.cpu().numpy() + np.asarray(art, dtype=np.float64)
