"""Ensembles sharded across GPUs: one process per GPU, systems partitioned by
cost (the FP64 step of a system costs about n^5), no communication while the
systems propagate, one gather of the per-step dipoles at the end.

No counterpart in the reference (it runs one system per process)."""
from __future__ import annotations

import heapq

import numpy as np


def partition(params, world):
    """Longest-processing-time assignment of systems to `world` ranks by the
    cost n^5; returns one sorted index list per rank."""
    cost = [float(p.Ns * p.Nb) ** 5 for p in params]
    order = sorted(range(len(params)), key=lambda i: (-cost[i], i))
    heap = [(0.0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + cost[i], r))
    return [sorted(x) for x in out]


def _gpu_propagate(params, nsteps, device):
    from . import Batch, make_G0
    if not params:
        return np.zeros((0, nsteps)), 0.0
    with Batch(params, "fp64", device) as b:
        for i, p in enumerate(params):
            b.set_state(i, make_G0(p))
        b.adiabatic_switch()
        dip = b.propagate(nsteps)
        return dip, b.last_device_ms


def run_sharded(params, nsteps, rank=0, world=1, device=0, group=None, propagate=None):
    """Every rank propagates its share of `params` (G0, adiabatic switching,
    nsteps RK4 steps) on `device`; rank 0 returns (dipoles [nsys][nsteps] in
    the order of `params`, max device ms over ranks), the other ranks
    (None, max ms).  `propagate(params, nsteps, device) -> (dipoles, ms)`
    replaces the GPU batch (tests)."""
    import torch
    import torch.distributed as dist
    shards = partition(params, world)
    mine = shards[rank]
    fn = propagate or _gpu_propagate
    dip, ms = fn([params[i] for i in mine], nsteps, device)
    dip = np.asarray(dip, np.float64).reshape(len(mine), nsteps)
    if world == 1:
        return dip, ms
    t = torch.tensor([ms], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    parts = [None] * world if rank == 0 else None
    dist.gather_object(dip, parts, dst=0, group=group)
    if rank != 0:
        return None, float(t.item())
    out = np.zeros((len(params), nsteps))
    for r, idx in enumerate(shards):
        out[idx] = parts[r]
    return out, float(t.item())
