"""The learned extrapolator's RK4 judge and fallback (learned.judged_rollout):
plain RK4 re-runs the judged trajectories, compares the dipole at every
checkpoint, and from the first failed checkpoint on every trajectory's output
is the RK4 trajectory."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(g12, L, torch, nsys=3, P=48):
    ps = L.window_params(nsys, seed=9, time_steps=400)
    pre, states = [], []
    for p in ps:
        f, st, _ = L.rk4_prefix(p, P, "bf16oz")
        pre.append(f)
        states.append(st)
    prefix = torch.from_numpy(np.stack(pre)).cuda()
    ex = L.Extrapolator(16, K=32, M=16, width=128, max_batch=128, seed=3)
    ex.fit_norm(prefix)
    return ps, states, prefix, ex


def test_untrained_network_falls_back_to_rk4(g12):
    torch = pytest.importorskip("torch")
    from g12kba_b200 import learned as L
    ps, states, prefix, ex = _setup(g12, L, torch)
    P, total = prefix.shape[1], 48 + 128
    out, rep = L.judged_rollout(ex, ps, states, prefix, total, check_every=32, tol=1e-3, judge=1, seed=0)
    assert rep["fallback"] and rep["accepted_after_prefix"] == 0 and len(rep["judged"]) == 1
    T = out.shape[1]
    for i, p in enumerate(ps):
        f, _, _ = L._rk4_features(p, states[i], T - P, "bf16oz", 0)
        assert np.array_equal(out[i, P:], f), i
        assert np.array_equal(out[i, :P], prefix[i].cpu().numpy())


def test_accepted_network_output_is_kept(g12):
    torch = pytest.importorskip("torch")
    from g12kba_b200 import learned as L
    ps, states, prefix, ex = _setup(g12, L, torch)
    P, total = prefix.shape[1], 48 + 128
    pred, _ = ex.rollout(prefix, total)
    out, rep = L.judged_rollout(ex, ps, states, prefix, total, check_every=32, tol=1e30, judge=None)
    assert not rep["fallback"] and rep["accepted_after_prefix"] == out.shape[1] - P
    assert rep["judged"] == [0, 1, 2] and rep["judge_rk4_ms"] > 0
    # the network's own snapshots (a separate rollout: split-K sums may differ in the last bits)
    pred = pred.cpu().numpy()
    assert np.array_equal(out[:, :P], prefix.cpu().numpy())
    assert np.max(np.abs(out - pred)) <= 1e-3 * np.max(np.abs(pred))
