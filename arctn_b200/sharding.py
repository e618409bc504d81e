"""Many independent networks across ranks: longest-processing-time-first sharding and one gather.

The networks of a batch share nothing, so a multi-GPU run needs no data-path collective: each rank takes a
share of the networks, runs them as its own ProgramBatch, and the per-network results are gathered once, in
network order.  Shares are balanced by work with the LPT rule (networks in decreasing cost, each to the rank
with the least work so far), whose largest share is at most 4/3 of the best possible one.  The reference has
no batch form; its scale-out of independent work is the MPI slice runner (src/bin/tnmpi.rs), whose single
collective this mirrors.
"""

from __future__ import annotations

import heapq
import math


def lpt_shard(costs, ranks):
    """Per-rank lists of item indices (each list ascending) for items of the given costs.  Items go in
    decreasing cost, ties by lower index, each to the rank with the least assigned cost, ties by lower rank,
    so the assignment is deterministic and the same on every rank."""
    ranks = int(ranks)
    if ranks < 1:
        raise ValueError(f"ranks must be positive, got {ranks}")
    costs = [float(c) for c in costs]
    if any(not (math.isfinite(c) and c >= 0) for c in costs):
        raise ValueError("costs must be finite and non-negative")
    heap = [(0.0, r) for r in range(ranks)]
    shares = [[] for _ in range(ranks)]
    for i in sorted(range(len(costs)), key=lambda j: (-costs[j], j)):
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(s) for s in shares]


def run_sharded(costs, execute_share, rank, ranks, gather=None):
    """Run this rank's LPT share and gather every network's result, in network order, on every rank.

    ``execute_share(indices)`` runs the given networks (ascending indices) and returns one result per index.
    ``gather(obj)`` returns the list of every rank's ``obj`` in rank order (``torch.distributed``'s
    ``all_gather_object`` by default), the run's one collective."""
    shares = lpt_shard(costs, ranks)
    mine = shares[rank]
    results = list(execute_share(mine)) if mine else []
    if len(results) != len(mine):
        raise ValueError(f"execute_share returned {len(results)} results for {len(mine)} networks")
    if gather is None:
        import torch.distributed as dist

        def gather(obj):
            out = [None] * ranks
            dist.all_gather_object(out, obj)
            return out

    everyone = gather(list(zip(mine, results)))
    out = [None] * len(costs)
    for part in everyone:
        for i, value in part:
            out[i] = value
    return out
