"""RK4 steps/s of the HF-GKBA G1-G2 propagation at Ns=16, Nb=2 (n=32) on B200.

Workload (the configuration the headline metric is quoted on): Hubbard chain
Ns=16, Nb=2, t1=1, t2=0.3, U=1.5, EHM with w(r)=U/(1+r), full quench 1.5 on
Nq=4 sites, dt=0.01.  Initial state: make_G0, then the adiabatic switching
phase (untimed); a "step" is one RK4 step (4 stages) of the propagation.

Arms:
  default            the library (C ABI via ctypes) on cuda:LOCAL_RANK; one
                     independent replica per rank ("replicas only": a single
                     system does not shard), value = all ranks' steps / max time.
  --impl reference   the reference's own OpenMP CPU build (oracle/_ref/g12_ref,
                     compiled from the reference headers) on the host cores,
                     RK4 steps of the same workload; rank 0 only.

Timing: device time of the K timed steps from CUDA events on the library's
stream (synchronised on both sides), max over ranks; the working set (2 x 5
tensors of 16 MB) exceeds the 126 MB L2.  e2e: the same K steps through the
C ABI from host buffers (state upload, per-step G1 snapshots copied back,
state download), wall clock.
"""
import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

WORKLOAD = dict(Ns=16, Nb=2, Nq=4, time_steps=10000, U=1.5, t1=1.0, t2=0.3, dt=0.01, EHM=True,
                v_law="inv", q_type="full", quench_strength=1.5)
METRIC = "RK4 steps/s at Ns=16,Nb=2: mixed/learned vs plain FP64 on B200, G1 err<=1e-6"
CONFIG = {"workload": "HF-GKBA GW, Hubbard chain Ns=16 Nb=2 (n=32), EHM w(r)=U/(1+r), U=1.5, t2=0.3, "
                      "full quench 1.5 on Nq=4, dt=0.01",
          "n": 32, "g2_entries_per_tensor": 32 ** 4,
          "l2_policy": "L2 flushed between timed steps: every step is timed on its own (CUDA events "
                       "around its graph) and followed by a 160 MiB device write outside the timed span; "
                       "the mixed engine's working set (85 MB) would otherwise stay in the 126 MB L2"}
EVICT_BYTES = 160 << 20


# DRAM bytes (read + write) per launch of the top kernels at n = 32, from one
# `ncu --set full` capture each (the profiles/ summaries give the command).
TOP_KERNEL_DRAM_BYTES = {
    "k_sym_gemm_oz2": 16856320.0,
    "k_sym_epi": 37164288.0,
    "k_apply_tc<cols+epilogue>": 170896896.0,
}

# Algorithmic HBM bytes per launch in units of n^4 (both G2 tensors):
#   k_sym_gemm_*: read the FP32 stage input (16 n^4), write W (16 n^4);
#   k_sym_epi:    read W (16), Yc (16.5), Ac (24.75 stage average), write the next
#                 FP32 input (16) and, at the last stage, Yc (16.5 / 4): 77.4 n^4.
ALG_BYTES_N4 = {"k_sym_gemm_oz2": 32.0, "k_sym_gemm_oz": 32.0, "k_sym_gemm_tc": 32.0, "k_sym_gemm_simt": 32.0,
                "k_sym_epi": 77.4}
MIXED_STEP_BYTES_N4 = 4 * (32.0 + 77.4)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        if shutil.which("nvidia-smi") is None:
            return self
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits", "-lms", "100"],
                                     stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        time.sleep(0.5)  # nvidia-smi's first sample
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def allmax(pg, v):
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def reference_cpu(steps, warmup, max_seconds=None):
    """Times the compiled reference (OpenMP, all host cores) on RK4 steps of the
    workload.  Returns (steps/s, cores, sample description, per-step seconds)."""
    from oracle import REF_EXE, Config
    cores = os.cpu_count() or 1
    cfg = Config(Ns=16, Nb=2, Nq=4, time_steps=10000, U=1.5, t1=1.0, t2=0.3, dt=0.01, EHM=True, vlaw="inv",
                 q_type="full", quench_strength=1.5)
    env = dict(os.environ, OMP_NUM_THREADS=str(cores))
    if not os.path.exists(REF_EXE):
        return None
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "input"), "w") as f:
            f.write(cfg.input_text())
        if max_seconds is not None:
            # size the sample: one step first, then as many as fit
            r = subprocess.run([REF_EXE, "--vlaw", "inv", "--time-rk", "0", "1"], cwd=d, env=env,
                               capture_output=True, text=True, check=True)
            one = json.loads(r.stdout.strip().splitlines()[-1])["seconds"]
            steps = int(max(2, min(steps, max_seconds / max(one, 1e-3))))
            warmup = 0
        r = subprocess.run([REF_EXE, "--vlaw", "inv", "--time-rk", str(warmup), str(steps)], cwd=d, env=env,
                           capture_output=True, text=True, check=True)
    js = json.loads(r.stdout.strip().splitlines()[-1])
    sps = js["rk_iterations"] / js["seconds"]
    sample = (f"{js['rk_iterations']} RK4 steps of the n=32 workload after {warmup} warm-up steps, "
              f"reference OpenMP build (oracle/_ref/g12_ref), OMP_NUM_THREADS={cores}")
    return sps, cores, sample, js["seconds"] / js["rk_iterations"]


def run_reference_arm(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # a bounded sample (about a minute of CPU work) of the K requested steps
    res = reference_cpu(args.steps, args.warmup, max_seconds=60.0)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": "compiled reference oracle/_ref/g12_ref not built"}))
        return
    sps, cores, sample, _ = res
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": sps, "unit": "steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / sps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (physics-defined input)",
        "config": dict(CONFIG, parallelism="OpenMP CPU, rank 0"),
        "cpu_baseline": {"value": sps, "unit": "steps/s", "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": sps, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def ensemble_measure(g12, local, rank=0, world=1, pg=None, steps=20, warmup=3, sample=16):
    """256 uneven systems (n = 4..24) in one batch per GPU (FP64 engine; with N
    ranks the systems are partitioned by cost, no communication while they
    propagate) against the same systems run one context at a time (a seeded
    sample of them on rank 0, scaled).  The ensemble's state (about 2 GB) is
    far larger than L2."""
    from g12kba_b200 import ensemble
    ps = g12.ensemble_params(256)
    mine = [ps[i] for i in ensemble.partition(ps, world)[rank]]
    with g12.Batch(mine, "fp64", local) as b:
        for i, p in enumerate(mine):
            b.set_state(i, g12.make_G0(p))
        b.propagate(warmup)
        barrier(pg)
        b.propagate(steps)
        ms = allmax(pg, b.last_device_ms)
    if rank != 0:
        return None
    rng = np.random.default_rng(1)
    idx = rng.choice(len(ps), size=sample, replace=False)
    seq_ms = 0.0
    for i in idx:
        with g12.Context(ps[i], "fp64", local) as ctx:
            ctx.set_state(g12.make_G0(ps[i]))
            ctx.propagate_dipole(warmup)
            ctx.propagate_dipole(steps)
            seq_ms += ctx.last_device_ms
    seq_total = seq_ms * len(ps) / sample
    ns = [p.n for p in ps]
    return {"systems": len(ps), "n_values": sorted(set(ns)), "ranks": world,
            "ensemble_steps_per_s": steps / (ms / 1e3), "system_steps_per_s": len(ps) * steps / (ms / 1e3),
            "one_context_at_a_time_steps_per_s_one_gpu": steps / (seq_total / 1e3),
            "speedup_vs_one_context_at_a_time": seq_total / ms,
            "note": f"{steps} timed steps after {warmup}, max device time over ranks; sequential figure from "
                    f"{sample} sampled systems x {len(ps)}/{sample} on one GPU; from G0 with G2 = 0 (step cost "
                    f"does not depend on the state)"}


def g2_exchange_asymmetry(X, Ns, Nb):
    """||G2 - e(G2)|| / ||G2||, e the particle exchange G2[mu2 mu1; nu2 nu1], for
    a tensor in the reference layout IDX_8D (commutators.h:60)."""
    n = Ns * Nb
    s, b = np.arange(n) % Ns, np.arange(n) // Ns
    i, j, k, l = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), np.arange(n), indexing="ij")  # mu1 mu2 nu1 nu2
    ref = (s[k] + s[l] * Ns + (b[k] + b[l] * Nb) * Ns * Ns + (s[i] + s[j] * Ns) * (Ns * Nb) ** 2 +
           (b[i] + b[j] * Nb) * Ns ** 4 * Nb ** 2)
    Y = X[ref]  # [mu1][mu2][nu1][nu2]
    return float(np.linalg.norm(Y - Y.transpose(1, 0, 3, 2)) / np.linalg.norm(Y))


def extended_model_measure(g12, local):
    """The extended model (Ns=8, Nb=2, n=16: t2=0.5, U=2, EHM w(r)=U/(1+r), pulse
    quench 2.0 on Nq=3 with rate 2 and on/off midpoints 15/25, dt=0.01, 5000 steps
    = 5001 iterations), the pulse switched on (quench_gate 0; the reference's t<50
    gate would keep it off for the whole run).  Every engine starts from the same
    switched state (the FP64 symmetric engine's adiabatic switching).  Errors
    against both FP64 engines: the plain one (the reference's algorithm) leaves
    the physical, exchange-symmetric states on this model (its G2's
    antisymmetric part grows from round-off), the symmetric one does not."""
    p = g12.make_params(Ns=8, Nb=2, Nq=3, U=2.0, t1=1.0, t2=0.5, dt=0.01, EHM=True, v_law="inv",
                        q_type="pulse", quench_strength=2.0, quench_rate=2.0, quench_on_midpoint=15.0,
                        quench_off_midpoint=25.0, time_steps=5000, quench_gate=0.0)
    T = g12.rk_iterations(p)
    with g12.Context(p, "fp64sym", local) as ctx:
        ctx.set_state(g12.make_G0(p))
        ctx.adiabatic_switch()
        S = ctx.get_state()
    out, trajs = {"iterations": T, "start": "FP64 symmetric engine's switched state"}, {}
    for prec in ("fp64", "fp64sym", "bf16oz", "tf32x3"):
        with g12.Context(p, prec, local) as ctx:
            ctx.set_state(*S)
            traj, rc = ctx.propagate(T)
            ms = ctx.last_device_ms
            _, XX, XY = ctx.get_state()
        trajs[prec] = traj
        out[prec] = {"steps_per_s": T / (ms / 1e3), "status": rc,
                     "g2_exchange_asymmetry_end": max(g2_exchange_asymmetry(XX, 8, 2), g2_exchange_asymmetry(XY, 8, 2))}
    for prec in ("fp64", "bf16oz", "tf32x3"):
        for refn in ("fp64sym", "fp64"):
            if prec == refn:
                continue
            ref, got = trajs[refn], trajs[prec]
            pr, pg = g12.dipole(ref), g12.dipole(got)
            out[prec][f"g1_max_rel_err_vs_{refn}"] = float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))
            out[prec][f"dipole_err_vs_{refn}"] = float(np.max(np.abs(pg - pr)) / max(np.max(np.abs(pr)), 1e-12))
    return out


def full_run_error(g12, p, S, precision, local):
    """The workload's full run (10,000 RK4 steps from the post-switching state
    S) on `precision` and on plain FP64; max G1 and dipole errors of the
    trajectory (error definitions of the tests: G1 relative to max |G1|,
    dipole relative to max |p|)."""
    T = g12.rk_iterations(p)
    out = {"iterations": T}
    trajs = {}
    for prec in ("fp64", precision):
        with g12.Context(p, prec, local) as ctx:
            ctx.set_state(*S)
            ctx.propagate(8)  # graph capture outside the timed call
            ctx.set_state(*S)
            t0 = time.perf_counter()
            tr, rc = ctx.propagate(T)
            wall = time.perf_counter() - t0
            out[prec + "_status"] = rc
            out[prec + "_device_s"] = ctx.last_device_ms / 1e3
            # the G1 snapshot of every step (T x n^2 complex) comes back during the call:
            # each finished half of the device ring is copied while the next half runs
            out[prec + "_call_wall_s"] = wall
            out[prec + "_snapshot_bytes"] = int(tr.nbytes)
        trajs[prec] = tr
    ref, got = trajs["fp64"], trajs[precision]
    out["g1_max_rel_err"] = float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))
    pr, pg_ = g12.dipole(ref), g12.dipole(got)
    out["dipole_max_rel_err"] = float(np.max(np.abs(pg_ - pr)) / max(np.max(np.abs(pr)), 1e-12))
    return out


def learned_measure(g12, local, ntrain=128, ntest=32, T=3000, P=150, train_steps=20000, check_every=200):
    """Learned extrapolator on its n=16 family (Ns=8, Nb=2, U ~ U[1,3],
    quench ~ U[0.5,3] switched on at t=1): trajectories from the batch engine,
    training on the GPU (windows from t = 1 on), rollout of held-out systems
    from an RK4 prefix of P steps (t = 1.5: past the quench midpoint), checked
    against their RK4 trajectories every `check_every` steps; the same network
    is also rolled out from a prefix of 400 steps."""
    import torch
    from g12kba_b200 import learned as L
    ps = L.window_params(ntrain + ntest, seed=5, time_steps=T)
    t0 = time.perf_counter()
    feat, _, gen_ms = L.generate(ps, T, stride=1, device=local)
    ok = L.stable(feat)
    okn = ok.cpu().numpy()
    ftr = feat[:ntrain][ok[:ntrain]].contiguous()
    fte = feat[ntrain:][ok[ntrain:]].contiguous()
    test_ps = [p for p, k in zip(ps[ntrain:], okn[ntrain:]) if k]
    del feat
    ex = L.Extrapolator(16, K=32, M=16, max_batch=512, seed=1)
    t1 = time.perf_counter()
    hist = ex.train(ftr, train_steps, batch=512, lr=1e-3, t_min=100)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t1
    pred, net_ms = ex.rollout(fte[:, :P], T)
    Tr = pred.shape[1]
    truth = fte[:, :Tr].cpu().numpy()
    pred = pred.cpu().numpy()
    errs = L.running_errors(pred, truth, 16, P - 1)
    h3, h2 = L.horizon(errs, 1e-3), L.horizon(errs, 1e-2)
    cks, ce = L.checkpoint_errors(pred, truth, 16, P - 1, check_every)
    # plain RK4 on one of these systems (FP64 and the mixed engine)
    rk = {}
    for prec in ("fp64", "bf16oz"):
        with g12.Context(test_ps[0], prec, local) as ctx:
            ctx.set_state(g12.make_G0(test_ps[0]))
            ctx.propagate_dipole(20)
            ctx.propagate_dipole(400)
            rk[prec] = 400 / (ctx.last_device_ms / 1e3)
    net_per_traj = (Tr - P) / (net_ms / 1e3)  # snapshots per second per trajectory (all rolled out together)
    # the non-learned comparator: exact DMD fitted on the same RK4 prefixes
    t2 = time.perf_counter()
    dmd = L.dmd_rollout(fte[:, :P], Tr, window=min(P - 1, 400))
    dmd_s = time.perf_counter() - t2
    derr = L.running_errors(dmd, truth, 16, P - 1)
    dt = 0.01

    def covered(h, prefix="fp64", P=P):
        # simulated time per second of "RK4 prefix + network within the horizon"
        return dt * (P + h) / (P / rk[prefix] + h / net_per_traj)

    # the same network from a longer prefix (400 steps)
    P4 = 400
    pred4, _ = ex.rollout(fte[:, :P4], T)
    err4 = L.running_errors(pred4.cpu().numpy(), fte[:, :pred4.shape[1]].cpu().numpy(), 16, P4 - 1)
    h34, h24 = L.horizon(err4, 1e-3), L.horizon(err4, 1e-2)
    prefix_400 = {"horizon_steps_median_err_le_1e-3": h34, "horizon_steps_median_err_le_1e-2": h24,
                  "speedup_vs_plain_fp64_within_1e-3": covered(h34, P=P4) / (dt * rk["fp64"]),
                  "mixed_prefix_speedup_vs_plain_fp64_within_1e-3": covered(h34, "bf16oz", P=P4) / (dt * rk["fp64"]),
                  "mixed_prefix_speedup_vs_plain_fp64_within_1e-2": covered(h24, "bf16oz", P=P4) / (dt * rk["fp64"])}

    # the product protocol: network extrapolation judged by plain RK4 at
    # checkpoints, RK4 fallback from the first failed checkpoint, every cost
    # counted (RK4 prefix, network, judge, fallback) - with every trajectory
    # judged, and with a seeded sample of 2 of them judged
    judged = {}
    nj = min(8, len(test_ps))
    pre, states, pre_ms = [], [], 0.0
    for p_ in test_ps[:nj]:
        f, st, ms_ = L.rk4_prefix(p_, P, "bf16oz", local)
        pre.append(f)
        states.append(st)
        pre_ms += ms_
    prefix = torch.from_numpy(np.stack(pre)).to(f"cuda:{local}")
    for tag, jn in (("all_judged", None), ("two_judged", 2)):
        _, rep = L.judged_rollout(ex, test_ps[:nj], states, prefix, 1000, check_every=check_every, tol=1e-3,
                                  judge=jn, precision="bf16oz", device=local)
        cost_s = (pre_ms + rep["network_ms"] + rep["judge_rk4_ms"] + rep["fallback_rk4_ms"]) / 1e3
        sim = nj * (rep["snapshots"] - 1) * dt
        judged[tag] = dict(rep, prefix_rk4_ms=pre_ms, simulated_time_per_s=sim / cost_s,
                           speedup_vs_plain_fp64=sim / cost_s / (dt * rk["fp64"]),
                           speedup_vs_plain_bf16oz=sim / cost_s / (dt * rk["bf16oz"]))

    return {
        "family": "Ns=8 Nb=2 (n=16), t2=0.5, EHM U/(1+r), U~U[1,3], full quench ~U[0.5,3] on Nq=3 at t=1, dt=0.01",
        "judged_rollout": judged,
        "train": {"trajectories": int(ftr.shape[0]), "steps_each": T, "windows_K_M": [32, 16],
                  "adam_steps": train_steps, "batch": 512, "seconds": train_s, "loss_first": float(hist[:20].mean()),
                  "loss_last": float(hist[-200:].mean()), "data_device_s": gen_ms / 1e3},
        "test_trajectories": int(fte.shape[0]), "rk4_prefix_steps": P,
        "network_rollout": {"snapshots_per_s_per_trajectory": net_per_traj,
                            "simulated_time_per_s_per_trajectory": dt * net_per_traj,
                            "device_ms": net_ms, "trajectories": int(fte.shape[0])},
        "plain_rk4_simulated_time_per_s": {k: dt * v for k, v in rk.items()},
        "horizon_steps_median_err_le_1e-3": h3, "horizon_steps_median_err_le_1e-2": h2,
        "check_every_steps": check_every,
        "dmd_comparator": {"horizon_steps_median_err_le_1e-3": L.horizon(derr, 1e-3),
                           "horizon_steps_median_err_le_1e-2": L.horizon(derr, 1e-2),
                           "median_err_after_200_steps": float(np.median(derr[:, min(199, derr.shape[1] - 1)])),
                           "host_seconds": dmd_s, "window": min(P - 1, 400)},
        "network_median_err_after_200_steps": float(np.median(errs[:, min(199, errs.shape[1] - 1)])),
        "checkpoint_median_err": {int(c): float(np.median(ce[:, i])) for i, c in enumerate(cks[:10])},
        "simulated_time_per_s_within_1e-3": covered(h3),
        "speedup_vs_plain_fp64_within_1e-3": covered(h3) / (dt * rk["fp64"]),
        "speedup_vs_plain_fp64_within_1e-2": covered(h2) / (dt * rk["fp64"]),
        "with_mixed_engine_prefix": {
            "note": "the RK4 prefix on the bf16oz engine (G1 within 1e-8 of FP64), then the network",
            "speedup_vs_plain_fp64_within_1e-3": covered(h3, "bf16oz") / (dt * rk["fp64"]),
            "speedup_vs_plain_fp64_within_1e-2": covered(h2, "bf16oz") / (dt * rk["fp64"])},
        "prefix_400": prefix_400,
        "wall_s": time.perf_counter() - t0,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="bf16oz", choices=["fp64", "tf32x3", "bf16oz", "tf32x6", "fp32"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-extended", action="store_true")
    ap.add_argument("--no-full-run", action="store_true")
    ap.add_argument("--no-writer", action="store_true")
    ap.add_argument("--skip-as", action="store_true",
                    help="start the timed steps from G0 (profiling runs); the cost of a step does not depend on the state")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference_arm(args)
        return

    world, rank, local, pg = dist_setup(args.gpus)
    import g12kba_b200 as g12
    p = g12.make_params(**WORKLOAD)
    n = p.n
    G0 = g12.make_G0(p)
    K = args.steps

    # plain FP64 path: prepared state S (adiabatic switching, untimed)
    fp = g12.Context(p, "fp64", local)
    fp.set_state(G0)
    if not args.skip_as:
        fp.adiabatic_switch()
    S = fp.get_state()
    fp.propagate_dipole(args.warmup)
    mixed = args.precision != "fp64"
    mx = g12.Context(p, args.precision, local) if mixed else fp
    if mixed:
        mx.set_state(*S)
        mx.propagate_dipole(args.warmup)

    # timed: K RK4 steps from S on each path (device time, CUDA events around each
    # step).  Between timed steps a write of EVICT_BYTES (> L2) evicts the state,
    # so every step finds it in HBM, not L2.
    for c in {id(fp): fp, id(mx): mx}.values():
        c.set_l2_eviction(EVICT_BYTES)
    barrier(pg)
    fp.set_state(*S)
    E_start = fp.total_energy()
    traj_fp, rc_fp = fp.propagate(K)
    ms_fp = allmax(pg, fp.last_device_ms)
    E_fp = fp.total_energy()
    barrier(pg)
    mx.set_state(*S)
    # clocks sampled over both timed runs of the mixed engine (the headline and
    # the L2-resident figure)
    with Clocks(local) as clk:
        traj_mx, rc = mx.propagate(K)
        dev_ms = mx.last_device_ms
        E_mx = mx.total_energy()
        barrier(pg)
        ms = allmax(pg, dev_ms)
        # the same steps without the eviction write (state L2-resident between steps)
        mx.set_l2_eviction(0)
        mx.set_state(*S)
        mx.propagate_dipole(K)
        ms_res = allmax(pg, mx.last_device_ms)
    value = world * K / (ms / 1e3)
    value_fp = world * K / (ms_fp / 1e3)
    g1_err = float(np.max(np.abs(traj_mx - traj_fp)) / np.max(np.abs(traj_fp)))
    launches = mx.launches_per_step * K

    # e2e through the C ABI with host buffers: the plain user call (no eviction
    # aid), every host buffer in pinned memory
    import ctypes

    import torch

    def pinned(shape):
        return torch.empty(shape, dtype=torch.complex128, pin_memory=True).numpy()

    dp = ctypes.POINTER(ctypes.c_double)
    ptr = lambda a: a.ctypes.data_as(dp)
    S_in = [pinned(a.shape) for a in S]
    for a, b in zip(S_in, S):
        a[...] = b
    S_out = [pinned(a.shape) for a in S]
    traj_host = pinned((K, n, n))
    done = ctypes.c_int64()
    L = g12.lib()
    barrier(pg)
    t0 = time.perf_counter()
    L.g12_set_state(mx.h, ptr(S_in[0]), ptr(S_in[1]), ptr(S_in[2]))
    L.g12_propagate(mx.h, K, ptr(traj_host), ctypes.byref(done))
    L.g12_get_state(mx.h, ptr(S_out[0]), ptr(S_out[1]), ptr(S_out[2]))
    t1 = time.perf_counter()
    e2e_s = allmax(pg, t1 - t0)
    assert done.value == K
    state_bytes = (n * n + 2 * n ** 4) * 16
    e2e = {"value": world * K / e2e_s, "unit": "steps/s", "h2d_bytes_per_step": state_bytes / K,
           "d2h_bytes_per_step": n * n * 16 + state_bytes / K,
           "note": f"g12_set_state + g12_propagate({K} steps, per-step G1 snapshots to host) + g12_get_state, "
                   "pinned host buffers, wall clock, as a user calls it (no L2 eviction between steps); the "
                   "state upload and download (33.5 MB each) are spread over the K steps"}
    # the reference's text output of a 10,000-step trajectory (write_to_file.h:52-69):
    # real_/imag_G1.txt, n^2 rows x T columns, 6 significant digits
    writer = None
    if rank == 0 and not args.no_writer:
        Tw = 10000
        big = np.tile(traj_host[: min(K, Tw)], (Tw // min(K, Tw) + 1, 1, 1))[:Tw]
        cwd = os.getcwd()
        with tempfile.TemporaryDirectory() as d:
            os.chdir(d)  # the reference writes real_/imag_<name> into the working directory
            try:
                t0 = time.perf_counter()
                rc_w = L.g12_write_cfile2D(b"G1.txt", ptr(big), Tw, n * n)
                tw = time.perf_counter() - t0
            finally:
                os.chdir(cwd)
            size = sum(os.path.getsize(os.path.join(d, f)) for f in os.listdir(d))
        writer = {"snapshots": Tw, "n": n, "seconds": tw, "bytes": size, "status": rc_w,
                  "threads": os.cpu_count(), "mb_per_s": size / tw / 1e6}

    # per-kernel device times (CUDA events around each launch on the library stream)
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {"hbm_gbs": 6650.0, "source": "fallback"}
    hbm = peaks.get("hbm_gbs", 6650.0)
    mx.set_l2_eviction(EVICT_BYTES)
    kt = mx.kernel_times(2)
    tot = sum(a * c for a, c in kt.values())
    kernels = {k: {"ms_per_launch": a, "launches_per_step": c, "share": a * c / tot} for k, (a, c) in kt.items()}
    top = max(kt, key=lambda k: kt[k][0] * kt[k][1])
    top_ms = kt[top][0]
    fp64_peak = g12.fp64_peak_tflops(local)
    if mixed:
        bytes_alg = ALG_BYTES_N4.get(top, 0.0) * n ** 4
        roofline = {"bound": "hbm", "kernel": top, "achieved": bytes_alg / (top_ms * 1e-3) / 1e9, "peak": hbm,
                    "unit": "GB/s", "frac": bytes_alg / (top_ms * 1e-3) / 1e9 / hbm,
                    "traffic": TOP_KERNEL_DRAM_BYTES.get(top), "algorithmic_bytes": bytes_alg,
                    "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum per launch from one ncu "
                                      "--set full capture of this kernel (profiles/), not measured in this run",
                    "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if "source" not in peaks else "fallback"}
    else:
        flops = 32.0 * n ** 5
        roofline = {"bound": "fp64", "kernel": top, "achieved": flops / (top_ms * 1e-3) / 1e12, "peak": fp64_peak,
                    "unit": "TFLOP/s", "frac": flops / (top_ms * 1e-3) / 1e12 / fp64_peak,
                    "traffic": TOP_KERNEL_DRAM_BYTES.get(top),
                    "peak_source": "measured FP64 FMA probe (g12_fp64_peak_tflops) on this GPU"}
    # whole step against the per-step figure 640 n^4 bytes (FP64 state passes)
    mb = MIXED_STEP_BYTES_N4 * n ** 4 if mixed else 640.0 * n ** 4
    step_roofline = {"bytes_per_step_fp64_state": 640.0 * n ** 4, "bytes_per_step_this_engine": mb,
                     "achieved_gbs": mb * value / world / 1e9, "frac_of_hbm": mb * value / world / 1e9 / hbm,
                     "flops_per_step": 256.0 * n ** 5, "fp64_peak_tflops": fp64_peak}
    # the plain FP64 engine's kernels: its top kernel against the measured FP64
    # peak (the two halves of the commutator: 16 n^5 real multiply-adds each)
    fp_kernels = None
    if mixed:
        fp.set_l2_eviction(EVICT_BYTES)
        kf = fp.kernel_times(2)
        totf = sum(a * c for a, c in kf.values())
        fp_kernels = {k: {"ms_per_launch": a, "launches_per_step": c, "share": a * c / totf} for k, (a, c) in kf.items()}
        topf = max(kf, key=lambda k: kf[k][0] * kf[k][1])
        tf = 32.0 * n ** 5 / (kf[topf][0] * 1e-3) / 1e12
        fp_kernels["roofline"] = {"bound": "fp64", "kernel": topf, "achieved": tf, "peak": fp64_peak,
                                  "unit": "TFLOP/s", "frac": tf / fp64_peak,
                                  "algorithmic_flops": 32.0 * n ** 5,
                                  "peak_source": "measured FP64 FMA probe (g12_fp64_peak_tflops) on this GPU"}
    if mixed:
        mx.close()
    fp.close()

    # the same timed steps on the FP64 symmetric engine (one contraction per
    # tensor and the compressed state, all in FP64): splits the mixed engine's
    # speed-up into its symmetry part and its precision part
    fp64sym = None
    if mixed and p.n in (8, 16, 32):
        with g12.Context(p, "fp64sym", local) as sy:
            sy.set_state(*S)
            sy.propagate_dipole(args.warmup)
            sy.set_l2_eviction(EVICT_BYTES)
            barrier(pg)
            sy.set_state(*S)
            traj_sy, rc_sy = sy.propagate(K)
            ms_sy = allmax(pg, sy.last_device_ms)
        fp64sym = {"value": world * K / (ms_sy / 1e3), "unit": "steps/s", "ms_per_step": ms_sy / K,
                   "status": rc_sy, "g1_max_rel_err_vs_fp64": float(np.max(np.abs(traj_sy - traj_fp)) /
                                                                    np.max(np.abs(traj_fp)))}

    # error of the full 10,000-step run of the workload (untimed): this engine
    # against plain FP64 from the same post-switching state
    full_run = None
    if mixed and rank == 0 and not args.no_full_run:
        full_run = full_run_error(g12, p, S, args.precision, local)

    sections = []

    def section(name, obj):
        # the large sub-results go on their own lines before the headline line
        if rank == 0 and obj is not None:
            print(json.dumps({"section": name, name: obj}), flush=True)
            sections.append(name)

    section("full_run", full_run)
    if not args.no_ensemble:
        section("ensemble", ensemble_measure(g12, local, rank, world, pg))
    if rank == 0 and not args.no_extended:
        section("extended_model_n16", extended_model_measure(g12, local))
    if rank == 0 and not args.no_learned:
        section("learned", learned_measure(g12, local))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        res = reference_cpu(8, 0, max_seconds=20.0)
        if res is not None:
            sps, cores, sample, _ = res
            cpu = {"value": sps, "unit": "steps/s", "cores": cores, "kind": "reference", "sample": sample}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if not mixed else args.precision,
            "data": "synthetic (physics-defined input: make_G0 + adiabatic switching)",
            "config": dict(CONFIG, precision=args.precision, parallelism=f"replicas x{world}"),
            "status": rc, "l2_resident": {"value": world * K / (ms_res / 1e3), "unit": "steps/s",
                                          "ms_per_step": ms_res / K},
            "plain_fp64": {"value": value_fp, "unit": "steps/s", "ms_per_step": ms_fp / K,
                           "status": rc_fp, "kernels": fp_kernels},
            "speedup_vs_plain_fp64": value / value_fp,
            "g1_max_rel_err_vs_fp64": g1_err,
            "fp64_symmetric": fp64sym,
            "full_run_err_vs_fp64": None if full_run is None else {
                k: full_run[k] for k in ("iterations", "g1_max_rel_err", "dipole_max_rel_err")},
            "energy": {"start": float(E_start[0]), "correlation_start": float(E_start[3]),
                       "fp64_rel_drift": float(abs(E_fp[0] - E_start[0]) / abs(E_start[0])),
                       "mixed_rel_drift": float(abs(E_mx[0] - E_start[0]) / abs(E_start[0])),
                       "correlation_change": float(E_mx[3] - E_start[3]),
                       "note": "g12_total_energy before and after the timed steps (constant U, quench masked)"},
            "e2e": e2e, "text_writer_n32_10k": writer, "gpu_launches": launches, "roofline": roofline, "step_roofline": step_roofline,
            "kernels": kernels, "cpu_baseline": cpu, "clocks": clk.summary(),
            "sections_printed_above": sections,
        }
        print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
