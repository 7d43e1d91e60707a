"""Ladders across GPUs (one process per GPU).

Temperature ladders are independent between their own replica exchanges, and
an exchange needs only the chi^2 of one ladder's rungs, so a ladder never
spans GPUs and the sampling loop has no collective. `partition` assigns whole
ladders to ranks, balancing the per-step cost of the fused step: per replica
the terms of the pairs and MS paths through the two sites over the k grid
plus the windowed transform (it does not grow with the supercell size, which
sets only the memory). `gather_summaries` is
the one collective, after sampling: every rank's per-ladder results (best
chi^2, acceptance, ...) end up on every rank in ladder order, through
torch.distributed (NCCL on GPUs, gloo on the CPU).
"""
from __future__ import annotations

import numpy as np


def ladder_cost(nrep, ncoord, ms_M, nk, nchan, nwin, ncoef):
    """Relative per-step cost of one ladder in the fused step: nrep replicas,
    each (4 ncoord pair terms + 2 ms_M path entries) over nk points plus
    nchan x nwin x ncoef transform taps."""
    return float(nrep) * ((4 * ncoord + 2 * ms_M) * nk + nchan * nwin * ncoef)


def partition(costs, world):
    """Greedy longest-first assignment of ladders to `world` ranks: returns a
    list (per rank) of ascending ladder indices, every ladder exactly once,
    loads within the largest single cost of each other."""
    costs = np.asarray(costs, float)
    order = np.argsort(-costs, kind="stable")
    load = np.zeros(world)
    parts = [[] for _ in range(world)]
    for i in order:
        r = int(np.argmin(load))
        parts[r].append(int(i))
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def gather_summaries(local, nladders, parts, group=None):
    """All-gather of per-ladder rows: `local` (len(parts[rank]), k) float64
    rows of this rank's ladders in parts[rank] order. Returns the
    (nladders, k) array in ladder order on every rank."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    local = np.ascontiguousarray(local, np.float64)
    k = local.shape[1]
    width = max(len(p) for p in parts)
    pad = np.full((width, k), np.nan)
    pad[:local.shape[0]] = local
    backend = dist.get_backend(group)
    dev = "cuda" if backend == "nccl" else "cpu"
    t = torch.from_numpy(pad).to(dev)
    out = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(out, t, group=group)
    res = np.full((nladders, k), np.nan)
    for r, p in enumerate(parts):
        rows = out[r].cpu().numpy()
        for q, li in enumerate(p):
            res[li] = rows[q]
    return res
