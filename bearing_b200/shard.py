"""Independent worlds across ranks: which worlds each rank takes.

A batch of independent worlds (many small Bearing worlds stepped together) shards with no exchange
between ranks: each rank steps its own worlds on its own GPU.  The work of a world's step grows
with its bodies and rows, so the worlds are dealt to balance that weight: heaviest first, each to
the rank with the least so far (the longest-processing-time rule, within 4/3 of the best split),
and each rank keeps its worlds in their original order.
"""
from __future__ import annotations

import heapq


def balance(weights, parts):
    """Splits world indices 0..len(weights)-1 into `parts` lists of similar total weight."""
    if parts < 1:
        raise ValueError("parts must be at least 1")
    loads = [(0.0, r) for r in range(parts)]
    heapq.heapify(loads)
    shards = [[] for _ in range(parts)]
    for i in sorted(range(len(weights)), key=lambda k: (-float(weights[k]), k)):
        load, r = heapq.heappop(loads)
        shards[r].append(i)
        heapq.heappush(loads, (load + float(weights[i]), r))
    return [sorted(s) for s in shards]


def shard_of(weights, rank, parts):
    """The world indices rank `rank` of `parts` takes."""
    if not 0 <= rank < parts:
        raise ValueError("rank must be in [0, parts)")
    return balance(weights, parts)[rank]
