"""Multi-GPU helpers.

A single solve does not shard: the merge tree funnels into one root merge,
so one process per GPU runs independent replicas.  A batch of independent
tridiagonals shards with no data-path collective: each rank solves its own
share of the instances.  The work of an instance grows like n^2 (the
secular sums of its upper merges), so shares balance sum n^2.
"""
from __future__ import annotations

from typing import List, Sequence

import numpy as np


def partition_instances(orders: Sequence[int], world: int) -> List[np.ndarray]:
    """Split instance indices over `world` ranks, balancing sum n^2 by the
    longest-processing-time rule (largest first, to the least-loaded rank;
    ties to the lower rank).  Deterministic; every index appears once; each
    rank's indices come back in ascending order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    orders = np.asarray(orders, dtype=np.int64)
    load = np.zeros(world, dtype=np.float64)
    parts: List[list] = [[] for _ in range(world)]
    for i in sorted(range(len(orders)), key=lambda j: (-int(orders[j]) ** 2, j)):
        r = int(np.argmin(load))
        parts[r].append(i)
        load[r] += float(orders[i]) ** 2
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def pack(offsets: Sequence[int], D: np.ndarray, E: np.ndarray, idx: Sequence[int]):
    """The instances `idx` of a packed batch as a packed batch of their own
    (offsets, D, E), in the layout brdc_dstebr_batched takes."""
    offsets = np.asarray(offsets, dtype=np.int64)
    orders = [int(offsets[i + 1] - offsets[i]) for i in idx]
    off = np.zeros(len(idx) + 1, dtype=np.int64)
    off[1:] = np.cumsum(orders)
    Dp = np.empty(int(off[-1]))
    Ep = np.zeros(int(off[-1]))
    for k, i in enumerate(idx):
        lo, hi = int(offsets[i]), int(offsets[i + 1])
        Dp[off[k]:off[k + 1]] = D[lo:hi]
        Ep[off[k]:off[k + 1] - 1] = E[lo:hi - 1]
    return off, Dp, Ep


def max_over_ranks(value: float, dist=None, device: str = "cpu") -> float:
    """The largest of every rank's `value` (a time: the job ends with its
    slowest rank); `dist` is torch.distributed or None for one process."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
