"""Sharding of independent operators (momentum sectors of one chain, disorder
instances) over the ranks of a ``torch.distributed`` process group, one rank
per GPU.

The operators of a batch share nothing during Lanczos: each rank builds and
solves only its own share, and the only exchange is the gather of the
results (a few doubles per operator) at the end — no collective on the data
path.  The share is a longest-processing-time bin packing of per-operator cost
estimates (dimension x (1 + off-diagonal hits per row)), so ranks finish
together even when the dimensions are uneven (the 924 ... 184,756-state
ensemble).  EDKit itself has no distributed path; this is the host logic
around ``batch_lanczos_e0`` / ``block_lanczos``.
"""
from __future__ import annotations

import heapq

import numpy as np


def partition(weights, nparts):
    """Longest-processing-time bin packing: indices of `weights` split into
    `nparts` lists with near-equal sums (each list in ascending index order).
    Deterministic, so every rank computes the same partition."""
    if nparts < 1:
        raise ValueError("partition: nparts must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i))
    heap = [(0.0, r) for r in range(nparts)]
    parts = [[] for _ in range(nparts)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(weights[i]), r))
    return [sorted(p) for p in parts]


def sharded_solve(specs, build, solve, weight=None, group=None):
    """Solve independent problems across the ranks of `group`.

    specs : list of picklable problem descriptions, identical on every rank
    build : spec -> operator (called only for this rank's share)
    solve : list of operators -> array of shape (len(share), k) (e.g. the
            lowest k eigenvalues from ``batch_lanczos_e0``)
    weight: spec -> cost estimate (default 1)

    Returns (results in the order of `specs`, this rank's indices).  Every
    rank receives the full results (one ``all_gather_object``).  Without an
    initialised process group the whole list is solved locally."""
    import torch.distributed as dist

    w = [1.0 if weight is None else float(weight(s)) for s in specs]
    dist_on = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size(group) if dist_on else 1
    rank = dist.get_rank(group) if dist_on else 0
    mine = partition(w, world)[rank]
    local = np.asarray(solve([build(specs[i]) for i in mine])) if mine else None
    if not dist_on or world == 1:
        return local, mine
    pieces = [None] * world
    dist.all_gather_object(pieces, (mine, local), group=group)
    out = None
    for idx, vals in pieces:
        if not idx:
            continue
        vals = np.asarray(vals)
        if out is None:
            out = np.full((len(specs),) + vals.shape[1:], np.nan, dtype=vals.dtype)
        out[idx] = vals
    return out, mine
