"""Work partitioning across GPUs (one process per GPU).

Trajectory pairs are independent, so the path shards without any exchange of
intermediate data: every rank computes its own share and only the small
results move.

* ``pair_shards``: split a paired batch into `world` contiguous index ranges
  of near-equal DP work (sum of L1*L2), in the given processing order.
* ``row_shards``: split the rows of an nq x nd matrix into `world` contiguous
  row blocks of near-equal work (sum of query lengths).
* ``max_over_ranks``: the timing rule for multi-GPU numbers (slowest rank).
* ``gather_rows``: assemble row blocks of a matrix on rank 0 (all-gather of
  the host results through the process group; used by drivers, not by the
  timed path).
"""
from __future__ import annotations

import numpy as np


def pair_cost(len_a, len_b) -> np.ndarray:
    return np.asarray(len_a, dtype=np.float64) * np.asarray(len_b, dtype=np.float64)


def _balanced_cuts(weights: np.ndarray, world: int) -> np.ndarray:
    """Cut points c_0=0 <= c_1 <= ... <= c_world=n with near-equal weight sums."""
    n = weights.shape[0]
    if world <= 1 or n == 0:
        return np.array([0, n], dtype=np.int64) if world <= 1 else np.zeros(world + 1, dtype=np.int64)
    cs = np.cumsum(weights)
    total = cs[-1]
    targets = total * np.arange(1, world) / world
    cuts = np.searchsorted(cs, targets, side="left") + 1
    cuts = np.clip(cuts, 0, n)
    return np.concatenate([[0], cuts, [n]]).astype(np.int64)


def pair_shards(len_a, len_b, world: int, order=None):
    """-> list of `world` int64 index arrays (into the pair list) covering every
    pair exactly once, each with about 1/world of the total L1*L2."""
    la = np.asarray(len_a)
    lb = np.asarray(len_b)
    idx = np.arange(la.shape[0], dtype=np.int64) if order is None else np.asarray(order, dtype=np.int64)
    cuts = _balanced_cuts(pair_cost(la[idx], lb[idx]), world)
    return [idx[cuts[r]:cuts[r + 1]] for r in range(world)]


def row_shards(q_len, world: int):
    """-> list of (start, end) row ranges of a Q x D matrix, near-equal work."""
    cuts = _balanced_cuts(np.asarray(q_len, dtype=np.float64), world)
    return [(int(cuts[r]), int(cuts[r + 1])) for r in range(world)]


def imbalance(weights, shards) -> float:
    """max shard work / mean shard work - 1."""
    w = np.asarray(weights, dtype=np.float64)
    loads = np.array([w[s].sum() for s in shards])
    return float(loads.max() / loads.mean() - 1.0) if loads.size and loads.mean() > 0 else 0.0


def max_over_ranks(value: float, device=None) -> float:
    """All-reduce MAX of a per-rank number (e.g. device milliseconds)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_rows(block: np.ndarray, rows: tuple, n_rows: int):
    """All-gather the (rows, block) pieces; rank 0 returns the assembled
    [n_rows, nd] matrix, other ranks None."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return block
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, (rows, block))
    if dist.get_rank() != 0:
        return None
    out = np.empty((n_rows, block.shape[1]), dtype=block.dtype)
    for (s, e), b in parts:
        out[s:e] = b
    return out
