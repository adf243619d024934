"""The learned extrapolator end to end on a small family: trajectories from the
batch engine, training on the GPU, rollout from an RK4 prefix, and what the
trained network gains over the method without it (holding the last RK4
snapshot) and over the untrained network, checked against the RK4 trajectory."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def family(g12):
    import torch
    from g12kba_b200 import learned as L
    ps = L.window_params(28, seed=21, time_steps=1200)
    feat, dip, _ = L.generate(ps, 1200, stride=1)
    ok = L.stable(feat).cpu().numpy()
    keep = torch.from_numpy(ok).cuda()
    feat = feat[keep].contiguous()
    assert feat.shape[0] >= 20
    return L, feat[:-4].contiguous(), feat[-4:].contiguous()


def test_trained_network_beats_no_network(family):
    L, ftr, fte = family
    n, P, H = 16, 400, 160
    ex = L.Extrapolator(n, K=32, M=16, max_batch=512, seed=3)
    hist = ex.train(ftr, 2500, batch=512, lr=1e-3, t_min=300)
    assert hist[-100:].mean() < 0.05 * hist[:20].mean()
    pred, ms = ex.rollout(fte[:, :P], P + H)
    truth = fte[:, :P + H].cpu().numpy()
    e_net = L.running_errors(pred.cpu().numpy(), truth, n, P - 1)
    e_hold = L.running_errors(L.naive_rollout(fte[:, :P], P + H).cpu().numpy(), truth, n, P - 1)
    raw = L.Extrapolator(n, K=32, M=16, max_batch=512, seed=3)
    raw.fit_norm(ftr, 300)
    e_raw = L.running_errors(raw.rollout(fte[:, :P], P + H)[0].cpu().numpy(), truth, n, P - 1)
    med = lambda e, s: float(np.median(e[:, s - 1]))  # running error after s steps
    # two blocks past the prefix: several times closer to RK4 than holding the
    # last RK4 snapshot or than the untrained network
    assert med(e_net, 32) < 0.25 * med(e_hold, 32), (med(e_net, 32), med(e_hold, 32))
    assert med(e_net, 32) < 0.25 * med(e_raw, 32), (med(e_net, 32), med(e_raw, 32))
    assert med(e_net, 16) < 1e-2
    # and still closer after 160 steps
    assert med(e_net, H) < 0.7 * med(e_hold, H), (med(e_net, H), med(e_hold, H))


def test_checkpoint_errors_bookkeeping(family):
    L, _, fte = family
    truth = fte.cpu().numpy()
    cks, e = L.checkpoint_errors(truth, truth, 16, 99, 200)
    assert list(cks[:3]) == [299, 499, 699] and np.all(e == 0)
