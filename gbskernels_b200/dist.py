"""Multi-GPU distribution of a batch: instances are independent, so a batch is
partitioned across ranks (one process per GPU) by cost, each rank evaluates its
shard with the single-GPU queue, and the (B,) results are gathered once.  No
collective touches the data path; torch.distributed carries only the final
gather of 16-byte results (and the bench's barrier / max-time reduction).

Cost model (per instance, relative): haf/lhaf 2^n n^3 (n = N/2), perm 2^(n-1) n,
tor 2^k k^2 (k modes).
"""

from __future__ import annotations

import heapq

import numpy as np


def instance_cost(func: str, dim: int) -> float:
    if func in ("haf", "lhaf"):
        n = (dim + 1) // 2
        return float(2 ** n) * max(n, 1) ** 3
    if func == "perm":
        return float(2 ** max(dim - 1, 0)) * max(dim, 1)
    if func == "tor":
        k = dim // 2
        return float(2 ** k) * max(k, 1) ** 2
    raise ValueError(func)


def shard(funcs, dims, world: int) -> list[list[int]]:
    """Greedy longest-processing-time partition of instances over `world` ranks.
    Returns, for every rank, the sorted instance indices it evaluates."""
    if world < 1:
        raise ValueError("world must be >= 1")
    costs = [instance_cost(f, d) for f, d in zip(funcs, dims)]
    order = sorted(range(len(costs)), key=lambda i: -costs[i])
    heap = [(0.0, r) for r in range(world)]
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(p) for p in parts]


def gather_results(local_idx, local_vals, total: int, group=None) -> np.ndarray:
    """All-gather every rank's (indices, values) and scatter into input order."""
    import torch.distributed as dist
    payload = (list(map(int, local_idx)), np.asarray(local_vals, dtype=np.complex128))
    got = [None] * dist.get_world_size(group)
    dist.all_gather_object(got, payload, group=group)
    out = np.full(total, np.nan + 1j * np.nan, dtype=np.complex128)
    for idx, vals in got:
        out[idx] = vals
    return out


def evaluate_sharded(funcs, mats, precisions=None, group=None) -> np.ndarray:
    """Evaluate a ragged mixed batch across the ranks of `group` (one GPU each)."""
    import torch.distributed as dist
    from . import Workspace
    precisions = precisions or ["fp64"] * len(mats)
    parts = shard(funcs, [m.shape[0] for m in mats], dist.get_world_size(group))
    mine = parts[dist.get_rank(group)]
    with Workspace() as ws:
        vals = ws.evaluate([funcs[i] for i in mine], [mats[i] for i in mine], [precisions[i] for i in mine])
    return gather_results(mine, vals, len(mats), group)
