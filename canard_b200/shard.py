"""Assignment of independent cases (the batched workload) to ranks.

Independent cases need no data exchange, so each rank advances its own subset
in one batched context; only the final metric is gathered. Cases are assigned
greedily by point count (largest first, each to the least loaded rank), which
is deterministic on every rank without communication.
"""
from __future__ import annotations

from typing import List, Sequence


def assign(npoints: Sequence[int], world: int) -> List[List[int]]:
    """Return, per rank, the indices of the cases it owns."""
    if world < 1:
        raise ValueError("world size must be positive")
    order = sorted(range(len(npoints)), key=lambda i: (-npoints[i], i))
    load = [0] * world
    owned: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owned[r].append(i)
        load[r] += npoints[i]
    for o in owned:
        o.sort()
    return owned


def my_cases(npoints: Sequence[int], world: int, rank: int) -> List[int]:
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return assign(npoints, world)[rank]
