"""Ragged instance batches across GPUs: one rank per GPU, instances partitioned by estimated
cost, no exchange during the anneals, one gather of the result records at the end.

The path shards over independent instances (an anneal never talks to another one), so the
only collectives are the gather of results and of each rank's failure, if any.  Costs follow
the engine's work model: an instance's Trotter step is sum over edges of 2|i - j| - 1 two-site
updates (the swap network of cuda/src/mps.cpp:126-145), each costing about cap^3 for the bond
cap cap = min(chi, 2^floor(n/2)) (the SVD of a 2cap x 2cap theta), over its schedule steps.
The partition is longest-processing-time first: instances in descending cost, each to the
rank with the least load so far (ties to the lower rank), which keeps the largest load within
4/3 of the optimum.  Every rank computes the same partition from the same inputs.
"""
from __future__ import annotations

import numpy as np


def instance_cost(p) -> float:
    """Estimated work of one anneal: updates per step x steps x cap^3."""
    d = np.abs(np.asarray(p.ej, np.int64) - np.asarray(p.ei, np.int64))
    per_step = float((2 * d[d > 0] - 1).sum())
    cap = 1
    while cap < p.chi and cap < (1 << (p.n // 2)):
        cap <<= 1
    cap = min(cap, p.chi)
    return max(per_step, 1.0) * max(p.steps, 1) * float(cap) ** 3


def partition(costs, world: int):
    """Instance indices per rank (each list in ascending index order), longest cost first."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def imbalance(costs, parts) -> float:
    """Largest rank load over the best any partition can do, max(mean rank load, largest
    instance) -- 1.0 means no partition is better."""
    loads = [sum(costs[i] for i in p) for p in parts]
    bound = max(sum(loads) / max(len(loads), 1), max(costs) if len(costs) else 0.0)
    return max(loads) / bound if bound > 0 else 1.0


class ShardError(RuntimeError):
    """Raised on every rank when any rank's shard failed; `failures` maps rank -> message."""

    def __init__(self, failures):
        super().__init__("; ".join(f"rank {r}: {m}" for r, m in sorted(failures.items())))
        self.failures = failures


def run_ragged(problems, runner=None, group=None, **kw):
    """Anneal a ragged batch across the ranks of the default process group (or `group`).

    Each rank runs its share with `runner(problems_of_this_rank, **kw)` -- by default
    ffi.anneal_batch, one batched launch sequence on this rank's GPU -- and all ranks gather
    the result records, so every rank returns the full list in the original order.  A rank
    whose runner raised contributes its message instead; then every rank raises ShardError
    together (no rank is left waiting in a collective).  Without an initialised process group
    this runs everything locally."""
    import torch.distributed as dist
    if runner is None:
        from . import ffi
        runner = ffi.anneal_batch
    if not (dist.is_available() and dist.is_initialized()):
        return list(runner(list(problems), **kw))
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    parts = partition([instance_cost(p) for p in problems], world)
    mine = parts[rank]
    try:
        res = list(runner([problems[i] for i in mine], **kw)) if mine else []
        payload = ("ok", list(zip(mine, res)))
    except Exception as exc:  # reported to every rank below
        payload = ("error", f"{type(exc).__name__}: {exc}")
    gathered = [None] * world
    dist.all_gather_object(gathered, payload, group=group)
    failures = {r: g[1] for r, g in enumerate(gathered) if g[0] != "ok"}
    if failures:
        raise ShardError(failures)
    out = [None] * len(problems)
    for _, pairs in gathered:
        for i, r in pairs:
            out[i] = r
    return out
