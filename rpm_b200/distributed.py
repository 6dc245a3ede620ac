"""Multi-GPU replicas: one process per GPU, independent trajectory shards.

Trajectories (vector x orientation x system) are independent, so the path
shards with no data-path collective: every rank propagates its own
contiguous block of trajectories, balanced by predicted cost (state dimension
x expected matvecs).  The only collectives are at the end: the maximum of the
per-rank device times (for whole-job throughput) and an all-gather of the
per-trajectory yields.  Works with the ``nccl`` backend on GPUs and ``gloo``
on CPU (tests).
"""

from __future__ import annotations

from typing import Sequence

import numpy as np


def shard_bounds(costs: Sequence[float], world: int) -> list[tuple[int, int]]:
    """Contiguous [start, end) blocks of trajectories, one per rank, with
    near-equal total cost (greedy prefix split on the cumulative cost)."""
    c = np.asarray(costs, dtype=float)
    if world < 1:
        raise ValueError("world size must be positive")
    if c.ndim != 1 or np.any(c < 0):
        raise ValueError("costs must be a 1-D array of nonnegative numbers")
    n = c.size
    cum = np.concatenate(([0.0], np.cumsum(c)))
    total = cum[-1]
    bounds, start = [], 0
    for r in range(world):
        if r == world - 1:
            end = n
        else:
            target = total * (r + 1) / world
            end = int(np.searchsorted(cum, target, side="left"))
            # pick the closer of the two cut points around the target
            if end > start and end <= n and abs(cum[end - 1] - target) < abs(cum[end] - target):
                end -= 1
            end = min(max(end, start), n)
        bounds.append((start, end))
        start = end
    return bounds


def trajectory_costs(dimensions: Sequence[int], expected_matvecs: Sequence[float] | None = None) -> np.ndarray:
    """Predicted cost per trajectory: state dimension x expected matvecs."""
    d = np.asarray(dimensions, dtype=float)
    m = np.ones_like(d) if expected_matvecs is None else np.asarray(expected_matvecs, dtype=float)
    return d * m


def max_over_ranks(value: float, dist, device=None) -> float:
    """Maximum of a per-rank scalar (e.g. the device time of the timed region)."""
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_yields(yields, dist, counts: Sequence[int] | None = None):
    """All-gather per-trajectory yields (1-D float64 tensors, possibly of
    different lengths per rank given by ``counts``) into one tensor in rank
    order."""
    import torch

    if dist is None or not dist.is_initialized():
        return yields
    world = dist.get_world_size()
    if counts is None:
        n = torch.tensor([yields.numel()], dtype=torch.int64, device=yields.device)
        sizes = [torch.zeros_like(n) for _ in range(world)]
        dist.all_gather(sizes, n)
        counts = [int(s.item()) for s in sizes]
    width = max(counts)
    padded = torch.zeros(width, dtype=yields.dtype, device=yields.device)
    padded[: yields.numel()] = yields
    parts = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded)
    return torch.cat([p[:k] for p, k in zip(parts, counts)])


def rank_shard(dimensions: Sequence[int], dist, expected_matvecs: Sequence[float] | None = None) -> tuple[int, int]:
    """This rank's contiguous [start, end) block of a trajectory list that
    every rank builds identically (cost-balanced by :func:`shard_bounds`)."""
    rank, world = (dist.get_rank(), dist.get_world_size()) if dist is not None and dist.is_initialized() else (0, 1)
    return shard_bounds(trajectory_costs(dimensions, expected_matvecs), world)[rank]


def propagate_sharded(propagator, states, system_index: Sequence[int], times_us, dist, *, lifetime_us: float,
                      dimensions: Sequence[int] | None = None):
    """Propagate this rank's shard of a trajectory list with a
    :class:`~rpm_b200.batched.BatchedPropagator` and all-gather the yields.

    ``states``/``system_index`` describe the whole job, identically on every
    rank; ``dimensions`` (default: each trajectory's system dimension) drives
    the cost balance.  Returns (this rank's BatchedResult or None when its
    shard is empty, (start, end), all yields in trajectory order)."""
    import torch

    idx = np.asarray(system_index)
    dims = (np.asarray([propagator.hamiltonians[int(k)].dimension for k in idx]) if dimensions is None
            else np.asarray(dimensions))
    start, end = rank_shard(dims, dist)
    result = None
    if end > start:
        result = propagator.propagate([states[k] for k in range(start, end)], times_us, system_index=idx[start:end],
                                      lifetime_us=lifetime_us)
        mine = torch.as_tensor(result.yields, dtype=torch.float64)
    else:
        mine = torch.zeros(0, dtype=torch.float64)
    if dist is not None and dist.is_initialized() and dist.get_backend() == "nccl":
        mine = mine.cuda()
    counts = None
    if dist is not None and dist.is_initialized():
        world = dist.get_world_size()
        counts = [e - s for s, e in shard_bounds(trajectory_costs(dims), world)]
    return result, (start, end), gather_yields(mine, dist, counts)
