"""Multi-GPU evaluation of a batch of independent image pairs: one process per GPU, pairs sharded
longest-processing-time first on an estimated cost, scores gathered on the host.

A pair is the unit of work and pairs never interact, so there is no collective on the data path:
each rank evaluates its shard with the single-GPU library and the only exchange is the gather of
the per-pair scores at the end (torch.distributed object gather, any backend).  The reference
evaluates one pair per process on one device (src/main.cpp:271-286); this is the batch form of
that loop.
"""
import heapq
import math

import numpy as np

from . import fsim_plane_size


def pair_cost(metric, w, h):
    """Relative cost of one w x h pair: the input bytes it reads (8 per pixel pair), plus for FSIM
    the transform work on its downscaled plane (34 complex 2-D transforms, 5 N log2 N each, at an
    assumed 4 flops per byte of input traffic)."""
    cost = 8.0 * w * h
    if metric == "fsim":
        w2, h2 = fsim_plane_size(w, h)
        n = w2 * h2
        cost += 34 * 5.0 * n * math.log2(max(2, n)) / 4.0
    return cost


def shard_lpt(costs, world):
    """Longest-processing-time-first assignment of items to `world` ranks.

    Returns one ascending index list per rank.  Items are taken in decreasing cost (ties by index)
    and each goes to the currently least-loaded rank (ties by rank), so the result is deterministic
    and every rank computes the same partition without communicating."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    shards = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(s) for s in shards]


def evaluate_sharded(evaluate, pairs, costs, rank, world, group=None):
    """Evaluates this rank's LPT shard of `pairs` with `evaluate(list_of_pairs) -> sequence of
    per-pair scores` and, for world > 1, gathers every rank's scores on every rank.

    Returns an array of all scores in the original pair order (rows: pairs; one column per score
    the metric produces)."""
    shards = shard_lpt(costs, world)
    mine = shards[rank]
    local = evaluate([pairs[i] for i in mine]) if mine else []
    local = [np.atleast_1d(np.asarray(s, dtype=np.float64)) for s in local]
    if world == 1:
        parts = [(mine, local)]
    else:
        import torch.distributed as dist
        parts = [None] * world
        dist.all_gather_object(parts, (mine, local), group=group)
    k = None
    for idx, vals in parts:
        if vals:
            k = len(vals[0])
            break
    out = np.full((len(pairs), k or 1), np.nan)
    for idx, vals in parts:
        for i, v in zip(idx, vals):
            out[i] = v
    return out
