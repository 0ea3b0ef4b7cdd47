"""CPU oracle of the per-vertex warm-start MLP (TEST INFRASTRUCTURE ONLY).

Forward, backward and AdamW of the 16 -> 64 -> 64 -> 1 ReLU network in FP64 numpy,
rounding to BF16 exactly where the GPU kernels do (inputs, the hidden activations fed to
the next layer, the weights, and the backward tiles staged for the weight-gradient
GEMMs), so the tensor-core kernels can be checked against it.  `fd_check` validates the
backward formulas themselves by central differences (no rounding).
"""
from __future__ import annotations

import numpy as np

IN, H = 16, 64
NFEAT = 10  # used inputs (the rest of the 16 are zero)
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * IN
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
P = OFF_B3 + 1


def bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def f32(x):
    return np.asarray(x, dtype=np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(H, IN), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3], p[OFF_B3])


def init_params(seed=3):
    """He-style initial weights (the same formula as dissolve_tp.mlp)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(P, dtype=np.float32)
    p[OFF_W1:OFF_B1] = rng.normal(0, np.sqrt(2.0 / NFEAT), H * IN)
    p[OFF_W1:OFF_B1].reshape(H, IN)[:, NFEAT:] = 0.0
    p[OFF_W2:OFF_B2] = rng.normal(0, np.sqrt(2.0 / H), H * H)
    p[OFF_W3:OFF_B3] = rng.normal(0, 0.1 / np.sqrt(H), H)
    return p


def features(U, Up, phi, ngphi, logD, k, mean, istd, opU=None, opDU=None):
    """Normalised inputs (rows = vertex * S + species), FP32 then BF16 as on the GPU:
    0 phi, 1 |grad phi|, 2 u^n, 3 u^{n-1}, 4 u^n - u^{n-1}, 5 log D, 6 k, 7 1,
    8 stiffness image of u^n, 9 of u^n - u^{n-1} (both (V, S) or None)."""
    V, S = U.shape
    rows = V * S
    x = np.zeros((rows, IN), dtype=np.float64)
    u = U.reshape(-1)
    up = Up.reshape(-1)
    vid = np.repeat(np.arange(V), S)
    sid = np.tile(np.arange(S), V)
    raw = [phi[vid] if phi is not None else np.zeros(rows),
           ngphi[vid] if ngphi is not None else np.zeros(rows),
           u, up, (U - Up).reshape(-1), np.asarray(logD)[sid], np.asarray(k)[sid]]
    raw += [None, np.zeros(rows) if opU is None else opU.reshape(-1),
            np.zeros(rows) if opDU is None else opDU.reshape(-1)]
    for f in range(NFEAT):
        if f == 7:
            continue
        x[:, f] = (f32(raw[f]) - f32(mean[f])) * f32(istd[f])
        x[:, f] = f32(x[:, f])
    x[:, 7] = 1.0
    return bf16(x)


def forward(p, X):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    W1, W2, w3 = bf16(W1), bf16(W2), bf16(w3)
    z1 = X @ W1.T + f32(b1)
    h1 = bf16(np.maximum(z1, 0.0))
    z2 = h1 @ W2.T + f32(b2)
    h2 = bf16(np.maximum(z2, 0.0))
    y = h2 @ w3 + f32(b3)
    return y, (z1, h1, z2, h2)


def loss_and_grad(p, X, T):
    """Mean squared error and its gradient with the GPU's BF16 staging points."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    W2b, w3b = bf16(W2), bf16(w3)
    y, (z1, h1, z2, h2) = forward(p, X)
    n = X.shape[0]
    e = y - T
    dy = (2.0 / n) * e
    g = np.zeros(P, dtype=np.float64)
    g[OFF_W3:OFF_B3] = h2.T @ dy
    g[OFF_B3] = dy.sum()
    dz2 = np.where(z2 > 0, dy[:, None] * w3b[None, :], 0.0)
    dz2b = bf16(dz2)
    dz1 = np.where(z1 > 0, dz2b @ W2b, 0.0)
    dz1b = bf16(dz1)
    g[OFF_W2:OFF_B2] = (dz2b.T @ h1).reshape(-1)
    g[OFF_B2:OFF_W3] = dz2b.sum(axis=0)
    g[OFF_W1:OFF_B1] = (dz1b.T @ X).reshape(-1)
    g[OFF_B1:OFF_W2] = dz1b.sum(axis=0)
    return float((e * e).sum()), g


def adamw(p, m, v, g, step, lr, b1=0.9, b2=0.999, eps=1e-8, wd=1e-4):
    p = np.asarray(p, dtype=np.float64).copy()
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    decay = np.ones(P, dtype=bool)
    decay[OFF_B1:OFF_W2] = decay[OFF_B2:OFF_W3] = False
    decay[OFF_B3] = False
    p -= lr * (mh / (np.sqrt(vh) + eps) + np.where(decay, wd * p, 0.0))
    return p, m, v


def _plain_loss(p, X, T):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    h1 = np.maximum(X @ W1.T + b1, 0.0)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0)
    y = h2 @ w3 + b3
    return float(((y - T) ** 2).mean())


def _plain_grad(p, X, T):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    z1 = X @ W1.T + b1
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0.0)
    y = h2 @ w3 + b3
    dy = 2.0 * (y - T) / X.shape[0]
    g = np.zeros(P)
    g[OFF_W3:OFF_B3] = h2.T @ dy
    g[OFF_B3] = dy.sum()
    dz2 = np.where(z2 > 0, dy[:, None] * w3[None, :], 0.0)
    dz1 = np.where(z1 > 0, dz2 @ W2, 0.0)
    g[OFF_W2:OFF_B2] = (dz2.T @ h1).reshape(-1)
    g[OFF_B2:OFF_W3] = dz2.sum(0)
    g[OFF_W1:OFF_B1] = (dz1.T @ X).reshape(-1)
    g[OFF_B1:OFF_W2] = dz1.sum(0)
    return g


def fd_check(seed=0, n=64, probes=40, h=1e-6):
    """Max relative error of the analytic gradient (no BF16) against central differences."""
    rng = np.random.default_rng(seed)
    p = init_params(seed).astype(np.float64)
    p[OFF_B1:OFF_W2] = rng.normal(0, 0.1, H)
    p[OFF_B2:OFF_W3] = rng.normal(0, 0.1, H)
    X = rng.normal(0, 1, (n, IN))
    X[:, 8:] = 0.0
    T = rng.normal(0, 1, n)
    g = _plain_grad(p, X, T)
    worst = 0.0
    for idx in rng.choice(np.flatnonzero(np.abs(g) > 1e-6), size=probes, replace=False):
        e = np.zeros(P)
        e[idx] = h
        fd = (_plain_loss(p + e, X, T) - _plain_loss(p - e, X, T)) / (2 * h)
        worst = max(worst, abs(fd - g[idx]) / max(abs(g[idx]), 1e-8))
    return worst
