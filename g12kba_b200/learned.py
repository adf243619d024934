"""Learned G1 extrapolator: a network trained on trajectories that the
propagation engine generates, mapping a window of K past G1 snapshots to the
next M snapshots.  No counterpart in the reference (G12KBA-GW has no learned
component); the RK4 propagation stays the check of its error and the fallback.

Training, inference and data generation all run on the GPU through the C ABI
(``g12_mlp_*``, ``g12_batch_propagate_features``); torch only provides device
buffers.  Snapshots are spaced ``stride`` RK4 steps apart.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import Batch, Context, G12Error, dipole, lib, make_G0, make_params

DEFAULT_DIMS = (8704, 512, 512, 512, 4352)


def _torch():
    import torch
    return torch


def features(G1):
    """rho = -i G1 [..., n, n] -> upper triangle (mu <= nu, row-major), real
    parts then imaginary parts (float32), the layout the kernels use."""
    G1 = np.asarray(G1)
    n = G1.shape[-1]
    iu = np.triu_indices(n)
    rho = -1j * G1[..., iu[0], iu[1]]
    return np.concatenate([rho.real, rho.imag], axis=-1).astype(np.float32)


def g1_from_features(f, n):
    """Inverse of features(): G1 = i rho with rho Hermitian."""
    f = np.asarray(f, np.float64)
    nt = n * (n + 1) // 2
    iu = np.triu_indices(n)
    rho = np.zeros(f.shape[:-1] + (n, n), np.complex128)
    rho[..., iu[0], iu[1]] = f[..., :nt] + 1j * f[..., nt:]
    rho = rho + np.conj(np.swapaxes(rho, -1, -2)) - np.eye(n) * np.real(rho[..., np.arange(n), np.arange(n)])[..., None]
    return 1j * rho


def dipole_from_features(f, n):
    """dipole.h:25-32 from features (Im G1_ii = Re rho_ii)."""
    f = np.asarray(f, np.float64)
    diag = np.array([i * n - i * (i - 1) // 2 for i in range(n)])
    d = f[..., diag]
    p = np.zeros(f.shape[:-1])
    for i in range(n // 2):
        p += 2.0 * (n / 2.0 - i - 0.5) * (d[..., i] - d[..., n - 1 - i]) / n
    return p


def window_params(nsys, seed, time_steps=6000, Ns=8, Nb=2):
    """The learned-extrapolator family: Ns=8, Nb=2 (n=16), t1=1, t2=0.5, EHM
    w(r)=U/(1+r), U ~ U[1,3], full quench of strength ~ U[0.5,3] on Nq=3 sites,
    dt=0.01.  The quench is switched on at t=1 (quench_gate 0, rate 0.2) so that
    the trajectories hold post-quench dynamics from their start."""
    rng = np.random.Generator(np.random.MT19937(seed))
    out = []
    for _ in range(nsys):
        U = float(rng.uniform(1.0, 3.0))
        qs = float(rng.uniform(0.5, 3.0))
        out.append(make_params(Ns=Ns, Nb=Nb, Nq=3, U=U, t1=1.0, t2=0.5, EHM=True, v_law="inv", dt=0.01,
                               time_steps=time_steps, q_type="full", quench_strength=qs, quench_gate=0.0,
                               quench_on_midpoint=1.0, quench_rate=0.2))
    return out


def generate(params, nsteps, stride=1, device=0):
    """Trajectories of every system (G0, adiabatic switching, nsteps RK4 steps)
    as snapshot features on the device: torch float32 [nsys][nsteps//stride][F],
    plus the per-step dipoles (numpy) and the device milliseconds."""
    torch = _torch()
    n = params[0].n
    F = n * (n + 1)
    snaps = nsteps // stride
    feat = torch.zeros((len(params), snaps, F), dtype=torch.float32, device=f"cuda:{device}")
    torch.cuda.synchronize()
    with Batch(params, "fp64", device) as b:
        for i, p in enumerate(params):
            b.set_state(i, make_G0(p))
        b.adiabatic_switch()
        dip = b.propagate_features(nsteps, stride, feat.data_ptr())
        ms = b.last_device_ms
    return feat, dip, ms


def stable(feat, bound=1.5):
    """Trajectories that stay finite with every density below `bound` (the
    reference's density guard, RK_solver.h:101-110, stops a run once
    2 Im G1_00 > 3); torch bool [ntraj]."""
    torch = _torch()
    return torch.isfinite(feat).all(dim=2).all(dim=1) & (feat.abs().amax(dim=(1, 2)) < bound)


class MLP:
    """The network (``g12_mlp``): FP32 master weights, bf16 tcgen05 GEMMs with
    FP32 accumulation, Adam."""

    def __init__(self, dims=DEFAULT_DIMS, max_batch=512, seed=0, device=0):
        self.dims = tuple(int(d) for d in dims)
        self.max_batch = max_batch
        self.device = device
        d = (C.c_int32 * 5)(*self.dims)
        h = C.c_void_p()
        rc = lib().g12_mlp_create(d, max_batch, seed, device, C.byref(h))
        if rc:
            raise G12Error(f"g12_mlp_create failed ({rc}): {lib().g12_mlp_last_error(None).decode()}")
        self.h = h

    def close(self):
        if self.h:
            lib().g12_mlp_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc):
        if rc:
            raise G12Error(f"libg12kba MLP error {rc}: {lib().g12_mlp_last_error(self.h).decode()}")

    @property
    def param_count(self):
        return int(lib().g12_mlp_param_count(self.h))

    def get_params(self):
        out = np.zeros(self.param_count, np.float32)
        self._chk(lib().g12_mlp_get_params(self.h, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def set_params(self, params):
        params = np.ascontiguousarray(params, np.float32)
        assert params.size == self.param_count
        self._chk(lib().g12_mlp_set_params(self.h, params.ctypes.data_as(C.POINTER(C.c_float))))

    def grads(self):
        out = np.zeros(self.param_count, np.float32)
        self._chk(lib().g12_mlp_get_grads(self.h, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def forward(self, X):
        """X: torch float32 (batch, dims[0]) on the device -> (batch, dims[4])."""
        torch = _torch()
        Y = torch.empty((X.shape[0], self.dims[4]), dtype=torch.float32, device=X.device)
        torch.cuda.synchronize()
        self._chk(lib().g12_mlp_forward(self.h, C.c_void_p(X.data_ptr()), X.shape[0], C.c_void_p(Y.data_ptr())))
        return Y

    def loss_grad(self, X, Y):
        _torch().cuda.synchronize()
        loss = C.c_double()
        self._chk(lib().g12_mlp_loss_grad(self.h, C.c_void_p(X.data_ptr()), C.c_void_p(Y.data_ptr()), X.shape[0],
                                          C.byref(loss)))
        return loss.value

    def adam(self, lr, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
        self._chk(lib().g12_mlp_adam(self.h, lr, beta1, beta2, eps, weight_decay))

    def set_norm(self, K, M, F, mean, s_in, s_abs, s_out):
        mean = np.ascontiguousarray(mean, np.float32)
        self._chk(lib().g12_mlp_set_norm(self.h, K, M, F, mean.ctypes.data_as(C.POINTER(C.c_float)), s_in, s_abs,
                                         s_out))

    def windows(self, feat, idx):
        torch = _torch()
        idx = np.ascontiguousarray(idx, np.int64)
        B = idx.shape[0]
        X = torch.zeros((B, self.dims[0]), dtype=torch.float32, device=feat.device)
        Y = torch.zeros((B, self.dims[4]), dtype=torch.float32, device=feat.device)
        torch.cuda.synchronize()
        self._chk(lib().g12_mlp_windows(self.h, C.c_void_p(feat.data_ptr()), feat.shape[0], feat.shape[1],
                                        idx.ctypes.data_as(C.POINTER(C.c_int64)), B, C.c_void_p(X.data_ptr()),
                                        C.c_void_p(Y.data_ptr())))
        return X, Y

    def train_windows(self, feat, idx, lr, weight_decay=0.0):
        idx = np.ascontiguousarray(idx, np.int64)
        loss = C.c_double()
        self._chk(lib().g12_mlp_train_windows(self.h, C.c_void_p(feat.data_ptr()), feat.shape[0], feat.shape[1],
                                              idx.ctypes.data_as(C.POINTER(C.c_int64)), idx.shape[0], lr,
                                              weight_decay, C.byref(loss)))
        return loss.value

    def grad_windows(self, feat, idx):
        """Loss and gradients of one batch of windows, no Adam step (the
        gradients are complete on the device when this returns)."""
        idx = np.ascontiguousarray(idx, np.int64)
        loss = C.c_double()
        self._chk(lib().g12_mlp_grad_windows(self.h, C.c_void_p(feat.data_ptr()), feat.shape[0], feat.shape[1],
                                             idx.ctypes.data_as(C.POINTER(C.c_int64)), idx.shape[0],
                                             C.byref(loss)))
        return loss.value

    def grad_tensor(self):
        """The device block of all gradients as a float32 torch tensor (a view:
        writes to it change the gradients the next Adam step uses)."""
        ptr, cnt = C.c_void_p(), C.c_int64()
        self._chk(lib().g12_mlp_grad_buffer(self.h, C.byref(ptr), C.byref(cnt)))

        class _View:
            __cuda_array_interface__ = {"shape": (cnt.value,), "typestr": "<f4", "data": (ptr.value, False),
                                        "version": 2}

        return _torch().as_tensor(_View(), device=f"cuda:{self.device}")

    def train_pushforward(self, feat, idx, r, lr, noise=0.0, weight_decay=0.0):
        idx = np.ascontiguousarray(idx, np.int64)
        loss = C.c_double()
        self._chk(lib().g12_mlp_train_pushforward(self.h, C.c_void_p(feat.data_ptr()), feat.shape[0], feat.shape[1],
                                                  idx.ctypes.data_as(C.POINTER(C.c_int64)), idx.shape[0], r, noise,
                                                  lr, weight_decay, C.byref(loss)))
        return loss.value

    def rollout(self, feat, t0):
        """Fill snapshots t0+1.. of every trajectory of feat (in place); device ms."""
        _torch().cuda.synchronize()
        ms = C.c_float()
        self._chk(lib().g12_mlp_rollout(self.h, C.c_void_p(feat.data_ptr()), feat.shape[0], feat.shape[1], t0,
                                        C.byref(ms)))
        return ms.value


def average_gradients(grad, pg=None):
    """In place: the mean of ``grad`` over the ranks of ``pg`` (all-reduce of
    the sum, then 1/world), the data-parallel step between the ranks'
    backward passes and their identical Adam steps."""
    import torch.distributed as dist
    world = dist.get_world_size(pg)
    if world > 1:
        dist.all_reduce(grad, op=dist.ReduceOp.SUM, group=pg)
        grad.mul_(1.0 / world)
    return grad


def broadcast_from_root(t, pg=None):
    """In place: rank 0's ``t`` on every rank of ``pg``."""
    import torch.distributed as dist
    if dist.get_world_size(pg) > 1:
        dist.broadcast(t, src=dist.get_global_rank(pg, 0) if pg is not None else 0, group=pg)
    return t


def train_data_parallel(mlp, feat, steps, lo, hi, pg=None, batch=512, lr=1e-3, lr_min=1e-5, weight_decay=0.0,
                        seed=0, log=None):
    """Data-parallel Adam over the ranks of ``pg``: every rank draws its own
    windows (t in [lo, hi)) from its own trajectories ``feat``, the gradients
    are averaged across ranks (one all-reduce of the gradient block per step)
    and every rank takes the same Adam step, so the parameters stay equal
    (rank 0's initial parameters are broadcast first).  ``mlp`` provides
    get_params / set_params / grad_windows / grad_tensor / adam.  Returns this
    rank's loss history."""
    import torch.distributed as dist
    torch = _torch()
    rank = dist.get_rank(pg)
    p0 = torch.as_tensor(np.asarray(mlp.get_params(), np.float32), device=feat.device)
    mlp.set_params(broadcast_from_root(p0, pg).cpu().numpy())
    rng = np.random.default_rng([seed, rank])
    ntraj = feat.shape[0]
    hist = []
    for it in range(steps):
        a = lr_min + 0.5 * (lr - lr_min) * (1 + math.cos(math.pi * it / max(1, steps)))
        idx = np.stack([rng.integers(0, ntraj, batch), rng.integers(lo, hi, batch)], axis=1)
        hist.append(mlp.grad_windows(feat, idx))
        g = average_gradients(mlp.grad_tensor(), pg)
        if g.is_cuda:
            torch.cuda.current_stream(g.device).synchronize()  # the reduction ran on torch's stream
        mlp.adam(a, weight_decay=weight_decay)
        if log and (it % max(1, steps // 20) == 0 or it == steps - 1):
            log(f"rank {rank} step {it} lr {a:.2e} loss {hist[-1]:.3e}")
    return np.array(hist)


class Extrapolator:
    """Window-to-future map over snapshot features: normalisation, training on
    device trajectories, rollout."""

    def __init__(self, n, K=32, M=16, width=512, max_batch=512, seed=0, device=0):
        self.n, self.K, self.M = n, K, M
        self.F = n * (n + 1)
        self.mlp = MLP((K * self.F, width, width, width, M * self.F), max_batch=max_batch, seed=seed, device=device)
        self.norm = None

    def fit_norm(self, feat, t_min=0):
        """Scales from the training trajectories: s_in / s_out = RMS of the
        window offsets / future offsets, s_abs = RMS deviation from the mean."""
        torch = _torch()
        f = feat[:, t_min:].double()
        mean = f.mean(dim=(0, 1))
        s_abs = float(torch.sqrt(((f - mean) ** 2).mean()))
        d_in = f[:, :-(self.K - 1)] - f[:, self.K - 1:]
        s_in = float(torch.sqrt((d_in ** 2).mean()))
        d_out = f[:, self.M:] - f[:, :-self.M]
        s_out = float(torch.sqrt((d_out ** 2).mean()))
        self.norm = (mean.float().cpu().numpy(), max(s_in, 1e-6), max(s_abs, 1e-6), max(s_out, 1e-6))
        self.mlp.set_norm(self.K, self.M, self.F, self.norm[0], self.norm[1], self.norm[2], self.norm[3])

    def train(self, feat, steps, batch=512, lr=1e-3, lr_min=1e-5, weight_decay=0.0, t_min=0, seed=0, log=None,
              pushforward=0, noise=0.0, warm=0.25, pg=None):
        """Adam on random windows (cosine learning-rate decay); after the first
        `warm` fraction of the steps, each step first rolls the network forward
        r ~ U{0..pushforward} blocks and trains on the windows it produced.
        With a process group ``pg`` every rank holds its own trajectories and
        the training is data-parallel (train_data_parallel; the normalisation
        is rank 0's).  Returns the loss history (one value per step)."""
        if pg is not None:
            if pushforward or noise:
                raise ValueError("data-parallel training covers plain windows (no pushforward, no noise)")
            torch = _torch()
            if self.norm is None:
                self.fit_norm(feat, t_min)
            v = torch.as_tensor(np.concatenate([self.norm[0], np.array(self.norm[1:], np.float32)]),
                                device=feat.device)
            v = broadcast_from_root(v, pg).cpu().numpy()
            self.norm = (v[:-3], float(v[-3]), float(v[-2]), float(v[-1]))
            self.mlp.set_norm(self.K, self.M, self.F, self.norm[0], self.norm[1], self.norm[2], self.norm[3])
            return train_data_parallel(self.mlp, feat, steps, max(self.K - 1, t_min), feat.shape[1] - self.M, pg,
                                       batch, lr, lr_min, weight_decay, seed, log)
        if self.norm is None:
            self.fit_norm(feat, t_min)
        rng = np.random.default_rng(seed)
        ntraj, snaps = feat.shape[0], feat.shape[1]
        lo = max(self.K - 1, t_min)
        hist = []
        for it in range(steps):
            a = lr_min + 0.5 * (lr - lr_min) * (1 + math.cos(math.pi * it / max(1, steps)))
            r = int(rng.integers(0, pushforward + 1)) if (pushforward and it >= warm * steps) else 0
            hi = snaps - (r + 1) * self.M  # the window plus r + 1 blocks fit
            idx = np.stack([rng.integers(0, ntraj, batch), rng.integers(lo, hi, batch)], axis=1)
            if r == 0 and noise == 0.0:
                hist.append(self.mlp.train_windows(feat, idx, a, weight_decay))
            else:
                hist.append(self.mlp.train_pushforward(feat, idx, r, a, noise, weight_decay))
            if log and (it % max(1, steps // 20) == 0 or it == steps - 1):
                log(f"step {it} lr {a:.2e} loss {hist[-1]:.3e}")
        return np.array(hist)

    def rollout(self, prefix, total):
        """prefix: torch float32 [ntraj][t0+1][F] of exact snapshots; returns
        ([ntraj][total][F] with snapshots t0+1.. predicted, device ms)."""
        torch = _torch()
        t0 = prefix.shape[1] - 1
        total = t0 + 1 + (total - t0 - 1) // self.M * self.M
        feat = torch.zeros((prefix.shape[0], total, self.F), dtype=torch.float32, device=prefix.device)
        feat[:, : t0 + 1] = prefix
        ms = self.mlp.rollout(feat, t0)
        return feat, ms


def _rk4_features(p, state, nsteps, precision, device):
    """nsteps RK4 steps of system p from `state` (G1, G2xx, G2xy) on a context
    of `precision`: (features [nsteps][F] float32 of the snapshots after each
    step, state after the steps, device ms)."""
    with Context(p, precision, device) as ctx:
        ctx.set_state(*state)
        traj, rc = ctx.propagate(nsteps + 1)  # snapshot s is the state before step s
        ms = ctx.last_device_ms
        st = ctx.get_state()
    if rc != 0:
        raise G12Error(rc, "RK4 stopped (density guard) during a judged rollout")
    return features(traj[1:]), st, ms


def rk4_prefix(p, nsnap, precision="bf16oz", device=0):
    """G0, adiabatic switching and nsnap - 1 RK4 steps of system p: the
    features of the nsnap snapshots (the switched state first), the exact
    state at the last of them and the device ms of the RK4 steps."""
    with Context(p, precision, device) as ctx:
        ctx.set_state(make_G0(p))
        ctx.adiabatic_switch()
        traj, rc = ctx.propagate(nsnap - 1)
        ms = ctx.last_device_ms
        st = ctx.get_state()
    if rc != 0:
        raise G12Error(rc, "RK4 stopped (density guard) in a prefix")
    return np.concatenate([features(traj), features(st[0])[None]]), st, ms


def judged_rollout(ex, params, prefix_states, prefix_feat, total, check_every=200, tol=1e-3, judge=None,
                   precision="bf16oz", device=0, seed=0):
    """Network extrapolation of an ensemble, judged by plain RK4.

    params: the systems; prefix_states: each system's exact state (G1, G2xx,
    G2xy) at the last prefix snapshot; prefix_feat: torch float32
    [nsys][P][F], the exact prefix snapshots (features); total: snapshots in
    the output.  The network rolls every trajectory out to `total`.  RK4 on the
    `precision` engine re-runs the judged trajectories (all, or a seeded sample
    of `judge` of them) from their prefix states and compares the dipole with
    the network's at every checkpoint (`check_every` snapshots); the network's
    snapshots count as accepted up to the last checkpoint at which every judged
    trajectory is within `tol` (dipole error relative to its RK4 maximum, the
    metric's definition).  From the first failed checkpoint on, RK4 is the
    fallback for every trajectory: the judged ones continue from their judge
    runs, the others run RK4 from their prefix states.

    Returns (features [nsys][total][F] numpy: network up to the accepted point,
    RK4 after it; a report with the accepted snapshots, the fallback flag, the
    judged systems and the device time of each part)."""
    torch = _torch()
    nsys, P = prefix_feat.shape[0], prefix_feat.shape[1]
    pred, net_ms = ex.rollout(prefix_feat, total)
    T = pred.shape[1]
    out = pred.cpu().numpy()
    n = ex.n
    rng = np.random.default_rng(seed)
    judged = np.arange(nsys) if judge is None or judge >= nsys else np.sort(rng.choice(nsys, judge, replace=False))
    rk_ms = 0.0
    rk_feat = {}
    for i in judged:
        f, _, ms = _rk4_features(params[i], prefix_states[i], T - P, precision, device)
        rk_feat[int(i)] = f
        rk_ms += ms
    # the judge on the device (g12_mlp_judge): running dipole error of every
    # judged trajectory at the checkpoints; accepted up to the last checkpoint
    # that all of them pass
    ref = pred[torch.as_tensor(judged, device=pred.device)].clone()
    for r, i in enumerate(judged):
        ref[r, P:] = torch.from_numpy(rk_feat[int(i)]).to(pred.device)
    sel = pred[torch.as_tensor(judged, device=pred.device)].contiguous()
    acc = np.zeros(len(judged), np.int64)
    torch.cuda.synchronize()
    ex.mlp._chk(lib().g12_mlp_judge(ex.mlp.h, C.c_void_p(sel.data_ptr()), C.c_void_p(ref.data_ptr()), len(judged),
                                    T, P - 1, check_every, tol, acc.ctypes.data_as(C.POINTER(C.c_int64))))
    # snapshots accepted after the prefix (the judge counts from snapshot P)
    accepted = int(acc.min())
    fallback = accepted < T - P
    fb_ms = 0.0
    if fallback:
        for i in range(nsys):
            if int(i) in rk_feat:
                f = rk_feat[int(i)]
            else:
                f, _, ms = _rk4_features(params[i], prefix_states[i], T - P, precision, device)
                fb_ms += ms
            out[i, P + accepted:] = f[accepted:]
    report = {"snapshots": T, "prefix": P, "accepted_after_prefix": accepted, "fallback": fallback,
              "judged": [int(i) for i in judged], "network_ms": net_ms, "judge_rk4_ms": rk_ms,
              "fallback_rk4_ms": fb_ms, "precision": precision, "tol": tol, "check_every": check_every}
    return out, report


def dipole_error(p, p_ref):
    """max_t |p - p_ref| / max(max_t |p_ref|, 1e-12) (the metric's definition)."""
    return float(np.max(np.abs(p - p_ref)) / max(np.max(np.abs(p_ref)), 1e-12))


def naive_rollout(prefix, total):
    """The method without a network past the exact prefix: hold the last
    snapshot (the comparator the tests measure the network's gain against)."""
    torch = _torch()
    out = torch.empty((prefix.shape[0], total, prefix.shape[2]), dtype=prefix.dtype, device=prefix.device)
    out[:, : prefix.shape[1]] = prefix
    out[:, prefix.shape[1]:] = prefix[:, -1:]
    return out


def checkpoint_errors(pred, truth, n, t0, every):
    """Dipole error of a rollout against the RK4 trajectory at the RK4
    checkpoints: for each checkpoint c (every `every` snapshots after t0),
    max over snapshots t0 < s <= c of |p - p_ref| / max|p_ref| (per trajectory).
    Returns (checkpoints, errors [ntraj][ncheck])."""
    pr = dipole_from_features(np.asarray(pred), n)
    pt = dipole_from_features(np.asarray(truth), n)
    amp = np.maximum(np.max(np.abs(pt), axis=1), 1e-12)
    e = np.maximum.accumulate(np.abs(pr[:, t0 + 1:] - pt[:, t0 + 1:]) / amp[:, None], axis=1)
    cks = np.arange(every, e.shape[1] + 1, every)
    return t0 + cks, e[:, cks - 1]


def horizon(errors_cum, tol):
    """Snapshots after the prefix for which the median running error stays <= tol."""
    med = np.median(errors_cum, axis=0)
    bad = np.nonzero(med > tol)[0]
    return int(bad[0]) if bad.size else int(med.size)


def running_errors(pred, truth, n, t0):
    pr = dipole_from_features(np.asarray(pred), n)
    pt = dipole_from_features(np.asarray(truth), n)
    amp = np.maximum(np.max(np.abs(pt), axis=1), 1e-12)
    return np.maximum.accumulate(np.abs(pr[:, t0 + 1:] - pt[:, t0 + 1:]) / amp[:, None], axis=1)


def dmd_rollout(prefix, total, window=400, rank=None, tol=1e-10):
    """Exact dynamic mode decomposition (Tu, Rowley, Luchtenburg, Brunton, Kutz,
    J. Comput. Dyn. 1, 2014) as the non-learned comparator: fit the linear map
    x_{s+1} = A x_s on the last `window` snapshots of each trajectory's exact
    prefix (numpy float64, host), in the basis of the singular vectors above
    `tol` (relative) or the first `rank`, and iterate it to `total` snapshots.
    prefix: [ntraj][t0+1][F] (numpy or torch); returns numpy [ntraj][total][F]."""
    pre = prefix.detach().cpu().numpy() if hasattr(prefix, "detach") else np.asarray(prefix)
    pre = pre.astype(np.float64)
    ntraj, t1, F = pre.shape
    out = np.zeros((ntraj, total, F))
    out[:, :t1] = pre
    for b in range(ntraj):
        Xw = pre[b, max(0, t1 - window - 1):t1].T  # F x (w+1)
        X, Y = Xw[:, :-1], Xw[:, 1:]
        U, sv, Vt = np.linalg.svd(X, full_matrices=False)
        r = int(np.sum(sv > tol * sv[0])) if rank is None else min(rank, sv.size)
        U, sv, Vt = U[:, :r], sv[:r], Vt[:r]
        At = U.T @ Y @ Vt.T / sv  # r x r, the map in the basis U
        z = U.T @ pre[b, -1]
        res = pre[b, -1] - U @ z  # the part outside the basis, held fixed
        for s_ in range(t1, total):
            z = At @ z
            out[b, s_] = U @ z + res
    return out
