"""One batch of independent matrices over several GPUs (one process per GPU).

The matrices of a batch need no communication while they are solved, so the batch is
partitioned: each rank takes a share chosen to balance the estimated cost, solves it
with the batched solver, and rank 0 gathers every matrix's INFO, SIGMA and the ranks'
device times back into the batch's order.  The cost of a matrix of order N is
estimated as N^4: one step costs N^3 (the pair weights' column scans dominate) and the
number of steps grows about linearly with N (the median measured on the 4096-matrix
workload is 9.4 N).  The share is the longest-processing-time rule: matrices in
decreasing cost, each to the rank with the least estimated cost so far, which bounds
a rank's total by 4/3 of the optimum.
"""
from __future__ import annotations

import numpy as np


def cost(n) -> np.ndarray:
    """Estimated relative cost of solving matrices of orders n."""
    return np.asarray(n, np.float64) ** 4


def partition(ns, world: int) -> list[np.ndarray]:
    """Indices of the batch (orders ns) for each of `world` ranks, by the
    longest-processing-time rule on cost(ns); each share in increasing index order."""
    ns = np.asarray(ns)
    c = cost(ns)
    order = np.argsort(-c, kind="stable")
    load = np.zeros(world)
    owner = np.empty(len(ns), np.int64)
    for m in order:
        r = int(np.argmin(load))  # the least-loaded rank, the lowest rank on ties
        owner[m] = r
        load[r] += c[m]
    return [np.nonzero(owner == r)[0] for r in range(world)]


def imbalance(shares, ns) -> float:
    """max rank cost / mean rank cost of a partition (1.0 = perfect balance)."""
    c = cost(ns)
    loads = np.array([c[s].sum() for s in shares])
    return float(loads.max() / loads.mean()) if loads.mean() > 0 else 1.0


def gather_results(share, results, count, group=None):
    """Rank 0 receives every rank's (indices, results) and returns the results in the
    batch's order (a list of `count` entries); the other ranks return None.  `results`
    are picklable per-matrix records in the order of `share`."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    payload = (np.asarray(share).tolist(), list(results))
    got = [None] * world if dist.get_rank(group) == 0 else None
    dist.gather_object(payload, got, dst=0, group=group)
    if got is None:
        return None
    out = [None] * count
    for idx, res in got:
        for i, r in zip(idx, res):
            out[i] = r
    return out


def solve_partitioned(mats, Js, solve, group=None):
    """Solve one batch over the ranks of the (initialised) process group: this rank's share
    by `solve(mats_share, Js_share) -> list of per-matrix records`, then the gather.
    Returns (all records in batch order on rank 0 / None elsewhere, this rank's share)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    ns = [np.asarray(Y).shape[0] for Y in mats]
    share = partition(ns, world)[rank]
    res = solve([mats[i] for i in share], [Js[i] for i in share]) if len(share) else []
    return gather_results(share, res, len(mats), group), share
