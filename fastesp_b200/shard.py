"""Points across GPUs: one process per GPU, points sharded, no collective on
the data path.

The ESP at a point depends on the pair table and that point only, so ranks
share nothing but the (replicated) table: every rank builds its table from the
same density and evaluates its own points.  Two layouts:

* weak scaling (``rank_points``): every rank its own point set of a fixed size
  (the benchmark's layout);
* strong scaling (``shard_range``/``esp_sharded``): one point set split into
  contiguous, balanced ranges, the values gathered where the caller wants them.

The only collectives are for bookkeeping: the maximum of per-rank timings
(``max_over_ranks``) and, in ``esp_sharded``, one all-gather of the results.
"""
from __future__ import annotations

import os

import numpy as np


def rank_info():
    """(rank, world size, local rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def shard_range(n: int, rank: int, world: int):
    """[start, stop) of rank's contiguous share of n points; sizes differ by <= 1."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of {world}")
    q, r = divmod(int(n), world)
    start = rank * q + min(rank, r)
    return start, start + q + (1 if rank < r else 0)


def rank_points(symbols, coords, n_points: int, rank: int, base_seed: int = 1):
    """This rank's own surface point set (weak scaling): seed base_seed + rank."""
    from .synth import vdw_surface_points
    return vdw_surface_points(symbols, coords, n_points, seed=base_seed + rank)


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank scalar (1-rank runs return it unchanged)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t[0])


def esp_sharded(evaluate, points, device=None):
    """Strong scaling: evaluate this rank's share of ``points`` with
    ``evaluate(points_share) -> values`` and all-gather the full result on
    every rank (in point order)."""
    import torch
    import torch.distributed as dist
    pts = np.asarray(points, np.float64).reshape(-1, 3)
    if not (dist.is_available() and dist.is_initialized()):
        return np.asarray(evaluate(pts), np.float64)
    rank, world = dist.get_rank(), dist.get_world_size()
    s0, s1 = shard_range(len(pts), rank, world)
    mine = torch.as_tensor(np.asarray(evaluate(pts[s0:s1]), np.float64), device=device)
    width = shard_range(len(pts), 0, world)[1]            # the largest share
    buf = torch.zeros(width, dtype=torch.float64, device=device)
    buf[: s1 - s0] = mine
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    out = []
    for r in range(world):
        a, b = shard_range(len(pts), r, world)
        out.append(parts[r][: b - a].cpu().numpy())
    return np.concatenate(out)
