"""The network oracle (numpy FP64) checked on its own: analytic gradients
against central finite differences, the bf16 rounding against torch's, and the
host-side feature helpers of the learned extrapolator."""
import numpy as np
import pytest

import oracle.mlp_oracle as mo


def _layers(rng, dims, scale=0.3):
    return [(scale * rng.standard_normal((dims[l + 1], dims[l])), 0.1 * rng.standard_normal(dims[l + 1]))
            for l in range(4)]


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    dims = (6, 5, 4, 5, 3)
    layers = _layers(rng, dims)
    X = rng.standard_normal((7, dims[0]))
    Y = rng.standard_normal((7, dims[4]))
    _, grads = mo.loss_grad(layers, X, Y, rounding=False)
    h = 1e-6
    for l in range(4):
        for which in (0, 1):
            P = layers[l][which]
            G = grads[l][which]
            for idx in list(np.ndindex(P.shape))[:6]:
                old = P[idx]
                P[idx] = old + h
                lp, _ = mo.loss_grad(layers, X, Y, rounding=False)
                P[idx] = old - h
                lm, _ = mo.loss_grad(layers, X, Y, rounding=False)
                P[idx] = old
                fd = (lp - lm) / (2 * h)
                assert abs(fd - G[idx]) <= 1e-6 * max(1.0, abs(fd)), (l, which, idx, fd, G[idx])


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(1)
    x = (rng.standard_normal(100000) * np.exp(rng.uniform(-20, 20, 100000))).astype(np.float32)
    ref = torch.from_numpy(x).to(torch.bfloat16).float().numpy().astype(np.float64)
    assert np.array_equal(mo.bf16(x), ref)


def test_feature_helpers_roundtrip_and_dipole(g12):
    from g12kba_b200 import learned
    rng = np.random.default_rng(2)
    n = 6
    a = rng.standard_normal((5, n, n)) + 1j * rng.standard_normal((5, n, n))
    G1 = 1j * (a + np.conj(np.swapaxes(a, -1, -2))) / 2
    f = learned.features(G1)
    assert f.shape == (5, n * (n + 1))
    assert np.allclose(f, mo.features(G1), atol=0)
    assert np.allclose(learned.g1_from_features(f, n), G1, atol=1e-6)
    assert np.allclose(learned.dipole_from_features(f, n), g12.dipole(G1), atol=1e-6)


def test_oracle_windows_layout():
    rng = np.random.default_rng(3)
    feat = rng.standard_normal((2, 40, 4))
    K, M = 4, 3
    mean = feat.mean(axis=(0, 1))
    X, Y = mo.windows(feat, [(1, 10)], K, M, mean, 2.0, 3.0, 5.0)
    assert X.shape == (1, K * 4) and Y.shape == (1, M * 4)
    assert np.allclose(X[0, :4], (feat[1, 7] - feat[1, 10]) / 2.0)
    assert np.allclose(X[0, 12:], (feat[1, 10] - mean) / 3.0)
    assert np.allclose(Y[0, 4:8], (feat[1, 12] - feat[1, 10]) / 5.0)


def test_dmd_reproduces_a_linear_system():
    """DMD on snapshots of x_{s+1} = A x_s (damped rotations) continues them exactly."""
    from g12kba_b200 import learned
    rng = np.random.default_rng(4)
    F, r = 40, 6
    Q, _ = np.linalg.qr(rng.standard_normal((F, F)))
    blocks = np.zeros((F, F))
    for k in range(r // 2):
        th, rho = 0.05 * (k + 1), 0.999 - 0.001 * k
        blocks[2 * k:2 * k + 2, 2 * k:2 * k + 2] = rho * np.array([[np.cos(th), -np.sin(th)], [np.sin(th), np.cos(th)]])
    A = Q @ blocks @ Q.T
    x = Q[:, :r] @ rng.standard_normal(r)
    traj = [x]
    for _ in range(499):
        traj.append(A @ traj[-1])
    traj = np.array(traj)[None]
    pred = learned.dmd_rollout(traj[:, :200], 500, window=150)
    assert np.max(np.abs(pred[0, 200:] - traj[0, 200:])) <= 1e-8 * np.max(np.abs(traj))


def test_particle_number_of_a_trajectory(g12):
    rng = np.random.default_rng(5)
    n = 6
    a = rng.standard_normal((3, n, n)) + 1j * rng.standard_normal((3, n, n))
    G1 = 1j * (a + np.conj(np.swapaxes(a, -1, -2))) / 2
    N = g12.particle_number(G1)
    assert np.allclose(N, 2 * np.trace(G1.imag, axis1=1, axis2=2))
