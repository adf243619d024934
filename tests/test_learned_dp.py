"""Data-parallel training of the extrapolator's network (host logic, CPU):
gradient averaging and the training loop over world_size-2 gloo process
groups.  The network is replaced by a linear least-squares stand-in with the
same interface (get/set_params, grad_windows, grad_tensor, adam), so no GPU is
needed; the GPU side of the interface is covered in tests/test_gpu_mlp.py."""
import os
import socket

import numpy as np
import torch
import torch.multiprocessing as mp

F, SNAPS, NTRAJ, STEPS, BATCH, LR = 6, 40, 5, 60, 16, 0.05
TRUE_W = torch.tensor([0.5, -1.0, 0.25, 2.0, 0.0, -0.75])


class LinearStandIn:
    """y = x . w fitted to x . TRUE_W (mean squared error)."""

    def __init__(self, seed):
        self.w = torch.tensor(np.random.default_rng(seed).standard_normal(F), dtype=torch.float32)
        self.g = torch.zeros(F)

    def get_params(self):
        return self.w.numpy().copy()

    def set_params(self, p):
        self.w = torch.tensor(np.asarray(p, np.float32))

    def grad_windows(self, feat, idx):
        idx = torch.as_tensor(idx)
        X = feat[idx[:, 0], idx[:, 1]]
        y = X @ TRUE_W
        r = X @ self.w - y
        self.g.copy_(2.0 * X.T @ r / X.shape[0])
        return float((r * r).mean())

    def grad_tensor(self):
        return self.g

    def adam(self, lr, weight_decay=0.0):
        self.w -= lr * self.g


def rank_feat(rank):
    return torch.tensor(np.random.default_rng(100 + rank).standard_normal((NTRAJ, SNAPS, F)), dtype=torch.float32)


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import torch.distributed as dist

    from g12kba_b200 import learned
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        g = torch.full((7,), float(rank + 1))
        learned.average_gradients(g)
        net = LinearStandIn(seed=rank)  # different initial parameters: rank 0's are broadcast
        hist = learned.train_data_parallel(net, rank_feat(rank), STEPS, 0, SNAPS - 1, None, BATCH, LR, LR, seed=3)
        q.put((rank, g.tolist(), net.get_params().tolist(), hist.tolist()))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _emulate(world):
    """The same training on one process: each step averages the ranks' gradients."""
    nets = [LinearStandIn(seed=0) for _ in range(world)]
    feats = [rank_feat(r) for r in range(world)]
    rngs = [np.random.default_rng([3, r]) for r in range(world)]
    for _ in range(STEPS):
        gs = []
        for r in range(world):
            idx = np.stack([rngs[r].integers(0, NTRAJ, BATCH), rngs[r].integers(0, SNAPS - 1, BATCH)], axis=1)
            nets[r].grad_windows(feats[r], idx)
            gs.append(nets[r].g.clone())
        mean = sum(gs) / world
        for n in nets:
            n.g.copy_(mean)
            n.adam(LR)
    return nets[0].get_params()


def test_data_parallel_training_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict((r, (g, w, h)) for r, g, w, h in (q.get(timeout=120) for _ in procs))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # gradient averaging: mean of 1 and 2 on both ranks
    assert out[0][0] == [1.5] * 7 and out[1][0] == [1.5] * 7
    # the parameters stay equal across ranks and follow the averaged gradients
    w0, w1 = np.array(out[0][1]), np.array(out[1][1])
    assert np.array_equal(w0, w1)
    assert np.allclose(w0, _emulate(2), rtol=1e-5, atol=1e-6)
    # and differ from what one rank learns from its own data alone
    assert not np.allclose(w0, _emulate(1), rtol=1e-3, atol=1e-4)
    for r in (0, 1):
        h = np.array(out[r][2])
        assert h[-10:].mean() < 0.5 * h[:10].mean()
