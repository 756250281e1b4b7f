"""Multi-GPU sharding of independent elections (one process per GPU).

Elections are independent, so a batch shards across ranks with no collective on the data
path: every rank builds the same deterministic work-balanced partition, closes its own share,
and only the small per-election results (rankings) are gathered at the end. The cost of an
election is its closure work, C^3 (padded to the 128-cell tile), plus its tally work
V * C^2 / 2 when ballots are included.
"""
from __future__ import annotations

import heapq
from typing import Sequence


def election_cost(C: int, V: int = 0, with_tally: bool = False) -> float:
    C = int(C)
    Cp = (C + 127) // 128 * 128
    # An election of at most 128 candidates is closed in one CTA, C pivot steps over a
    # 128 x 128 tile; larger ones pay for their padded tiles.
    cost = float(C) * 128 * 128 if C <= 128 else float(Cp) ** 3
    if with_tally:
        cost += float(V) * C * C / 2
    return cost


def partition_by_work(costs: Sequence[float], world: int) -> list[list[int]]:
    """Longest-processing-time greedy: elections in decreasing cost, each to the currently
    lightest rank (ties to the lowest rank). Deterministic, so every rank computes the same
    partition without communicating. Returns the election indices of each rank, ascending."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(p) for p in parts]


def gather_results(local: dict, world: int, group=None) -> dict | None:
    """Collects {election index: result} from every rank onto rank 0 (None elsewhere).
    Uses torch.distributed object collectives: gloo on CPU, NCCL on GPUs."""
    import torch.distributed as dist

    if world == 1:
        return dict(local)
    out = [None] * world if dist.get_rank(group) == 0 else None
    dist.gather_object(local, out, dst=0, group=group)
    if out is None:
        return None
    merged: dict = {}
    for part in out:
        overlap = merged.keys() & part.keys()
        if overlap:
            raise RuntimeError(f"elections {sorted(overlap)[:5]} closed on two ranks")
        merged.update(part)
    return merged
