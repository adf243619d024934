"""CPU oracle of the learned G1 extrapolator's network (test infrastructure only:
the tests use it to check the GPU training kernels; nothing in the product
imports it).

The reference (G12KBA-GW) has no learned component, so there is no reference
file to follow; this restates, in numpy FP64, the network the library trains
(g12kba_b200/csrc/mlp.cu) with the same operand rounding:

  forward   Z_l = bf16(A_{l-1}) bf16(W_l)^T + b_l,  A_l = gelu(Z_l) (l < 3),  A_3 = Z_3
  loss      mean((A_3 - Y)^2)
  backward  dZ_3 = 2 (A_3 - Y) / count
            dW_l = bf16(dZ_l)^T bf16(A_{l-1}),  db_l = sum_rows dZ_l
            dA_{l-1} = bf16(dZ_l) bf16(W_l),    dZ_{l-1} = dA_{l-1} * gelu'(Z_{l-1})

with A_{-1} = X, exact GELU 0.5 x (1 + erf(x / sqrt 2)), and bf16() the
round-to-nearest-even rounding of the FP32 value to bf16.  The GPU keeps
activations in FP32 and accumulates in FP32; the oracle accumulates in FP64,
so the two agree to FP32 accumulation error.
"""
import math

import numpy as np

_erf = np.vectorize(math.erf, otypes=[np.float64])


def bf16(x, enabled=True):
    """Round to bf16 (nearest even) through FP32, returned as float64
    (enabled=False: no rounding at all, for finite-difference checks)."""
    if not enabled:
        return np.asarray(x, dtype=np.float64)
    x32 = np.asarray(x, dtype=np.float32)
    u = x32.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def unpack(params, dims):
    """Flat FP32 parameter vector (per layer W [out][in], then b) -> [(W, b)]."""
    out, o = [], 0
    for l in range(4):
        nw = dims[l] * dims[l + 1]
        W = np.asarray(params[o:o + nw], np.float64).reshape(dims[l + 1], dims[l])
        o += nw
        b = np.asarray(params[o:o + dims[l + 1]], np.float64)
        o += dims[l + 1]
        out.append((W, b))
    return out


def pack(layers):
    return np.concatenate([np.concatenate([W.reshape(-1), b]) for W, b in layers])


def forward(layers, X, rounding=True):
    A = np.asarray(X, np.float64)
    Zs, As = [], [A]
    for l, (W, b) in enumerate(layers):
        Z = bf16(A, rounding) @ bf16(W, rounding).T + b
        Zs.append(Z)
        A = gelu(Z) if l < 3 else Z
        As.append(A)
    return Zs, As


def loss_grad(layers, X, Y, rounding=True):
    """(loss, [(dW, db)]) of the mean squared error."""
    Zs, As = forward(layers, X, rounding)
    Yh = As[-1]
    count = Yh.size
    loss = float(np.mean((Yh - Y) ** 2))
    dZ = 2.0 * (Yh - Y) / count
    grads = [None] * 4
    for l in range(3, -1, -1):
        W, _ = layers[l]
        Ain = As[l]
        dW = bf16(dZ, rounding).T @ bf16(Ain, rounding)
        db = dZ.sum(axis=0)
        grads[l] = (dW, db)
        if l == 0:
            break
        dA = bf16(dZ, rounding) @ bf16(W, rounding)
        dZ = dA * gelu_grad(Zs[l - 1])
    return loss, grads


def features(G1):
    """Snapshot features of G1 [..., n, n]: rho = -i G1, upper triangle
    (mu <= nu, row-major), real parts then imaginary parts."""
    G1 = np.asarray(G1)
    n = G1.shape[-1]
    iu = np.triu_indices(n)
    rho = -1j * G1[..., iu[0], iu[1]]
    return np.concatenate([rho.real, rho.imag], axis=-1)


def windows(feat, idx, K, M, mean, s_in, s_abs, s_out):
    """Network inputs and targets of windows (trajectory, t) of feat [traj][snap][F]."""
    X, Y = [], []
    for tr, t in idx:
        f = feat[tr]
        xt = f[t]
        slots = [(f[t - K + 1 + k] - xt) / s_in for k in range(K - 1)] + [(xt - mean) / s_abs]
        X.append(np.concatenate(slots))
        if t + M < f.shape[0]:
            Y.append(np.concatenate([(f[t + 1 + m] - xt) / s_out for m in range(M)]))
    return np.array(X), (np.array(Y) if Y else None)
