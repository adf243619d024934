"""Ensemble sharding across ranks (host logic, CPU): cost-balanced partition
and the end-of-run gather, with world_size-2 gloo process groups; the GPU batch
is replaced by a deterministic stand-in so no GPU is needed."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _fake_propagate(params, nsteps, device):
    # deterministic per-system "dipole": depends on the system only
    out = np.array([[p.U * (s + 1) + p.quench_strength + p.Ns * p.Nb for s in range(nsteps)] for p in params])
    return out.reshape(len(params), nsteps), float(len(params))


def _worker(rank, world, port, nsys, nsteps, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import torch.distributed as dist

    import g12kba_b200 as g12
    from g12kba_b200 import ensemble
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ps = g12.ensemble_params(nsys, time_steps=nsteps)
        dip, ms = ensemble.run_sharded(ps, nsteps, rank, world, propagate=_fake_propagate)
        q.put((rank, None if dip is None else dip.tolist(), ms))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_partition_balances_cost(g12):
    from g12kba_b200 import ensemble
    ps = g12.ensemble_params(256)
    for world in (1, 2, 4, 8):
        shards = ensemble.partition(ps, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(256))
        loads = [sum(float(ps[i].Ns * ps[i].Nb) ** 5 for i in s) for s in shards]
        assert max(loads) <= 1.05 * (sum(loads) / world) + max(float(p.Ns * p.Nb) ** 5 for p in ps)


def test_sharded_gather_matches_single_rank(g12):
    from g12kba_b200 import ensemble
    nsys, nsteps = 24, 5
    ps = g12.ensemble_params(nsys, time_steps=nsteps)
    ref, _ = ensemble.run_sharded(ps, nsteps, 0, 1, propagate=_fake_propagate)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, nsys, nsteps, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r, dip, ms = q.get(timeout=120)
        res[r] = (dip, ms)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[1][0] is None
    assert np.array_equal(np.array(res[0][0]), ref)
    # the time is the max over ranks
    shards = ensemble.partition(ps, 2)
    assert res[0][1] == res[1][1] == max(len(s) for s in shards)
