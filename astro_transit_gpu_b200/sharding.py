"""Multi-GPU plumbing: curves are independent, so a batch is split across
ranks (one process per GPU) with no data-path collective.

* ``lpt_assign``      longest-processing-time split of curves by cost
                      (points x periods), the balance rule for ragged batches
* ``max_over_ranks``  the job's device time: the slowest rank's (all-reduce MAX)
* ``gather_best``     optional all-gather of the fixed-size best-peak records,
                      when one rank needs every curve's result

The collectives go through ``torch.distributed`` (NCCL on GPUs, gloo on CPU);
nothing here touches another GPU's memory.
"""
from __future__ import annotations

import heapq
from typing import List, Optional, Sequence

import numpy as np


def lpt_assign(costs: Sequence[float], n_ranks: int) -> List[np.ndarray]:
    """Split curve indices over `n_ranks` by the LPT rule: curves in
    decreasing cost, each to the currently least-loaded rank (ties to the
    lowest rank).  Deterministic; every rank computing it gets the same split.
    The largest load is at most 4/3 of the optimum."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    costs = np.asarray(costs, dtype=np.float64)
    order = np.argsort(-costs, kind="stable")
    heap = [(0.0, r) for r in range(n_ranks)]
    parts: List[List[int]] = [[] for _ in range(n_ranks)]
    for c in order:
        load, r = heapq.heappop(heap)
        parts[r].append(int(c))
        heapq.heappush(heap, (load + float(costs[c]), r))
    return [np.sort(np.asarray(p, dtype=np.int64)) for p in parts]


def max_over_ranks(x: float, device=None, group=None) -> float:
    """The maximum of `x` over the ranks of the default (or given) process
    group; `x` itself without an initialised group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    v = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(v, op=dist.ReduceOp.MAX, group=group)
    return float(v.item())


def gather_best(best: np.ndarray, device=None, group=None) -> np.ndarray:
    """All-gather of per-curve best-peak records: `best` is a float64 array
    [n_local, k] (the same k on every rank, n_local may differ); returns the
    concatenation over ranks in rank order."""
    import torch
    import torch.distributed as dist
    best = np.ascontiguousarray(best, dtype=np.float64)
    if not (dist.is_available() and dist.is_initialized()):
        return best
    world = dist.get_world_size(group)
    k = best.shape[1]
    n = torch.tensor([best.shape[0]], dtype=torch.int64, device=device)
    ns = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(ns, n, group=group)
    n_max = max(int(v.item()) for v in ns)
    buf = torch.zeros((n_max, k), dtype=torch.float64, device=device)
    buf[:best.shape[0]] = torch.as_tensor(best, device=device)
    outs = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(outs, buf, group=group)
    return np.concatenate([o[:int(m.item())].cpu().numpy() for o, m in zip(outs, ns)])


def shard_of(costs: Sequence[float], rank: int, world: int) -> np.ndarray:
    """This rank's curve indices under ``lpt_assign``."""
    if not 0 <= rank < world:
        raise ValueError("rank outside [0, world)")
    return lpt_assign(costs, world)[rank]


def rank_seed(base: int, rank: Optional[int]) -> int:
    """Seed of a rank's synthetic batch under weak scaling (each rank searches
    its own curves)."""
    return int(base) + int(rank or 0)
