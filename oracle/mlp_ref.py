"""FP64 numpy restatement of the surrogate MLP -- TEST INFRASTRUCTURE ONLY (the checker
of the library's BF16 forward/backward kernels; never called by the product).

Network (parameter blob layout of mcs_surrogate_get_params):
  x = (features - mean) / std, padded 20 -> 32 with zeros
  h1 = silu(x W1 + b1), h2 = silu(h1 W2 + b2), h3 = silu(h2 W3 + b3)
  out = h3 W4 + b4 (16 columns, the first two used): mu = out[:, 0], s = clip(out[:, 1])
  loss = mean(s + (y - mu)^2 exp(-2 s) / 2)          (Gaussian NLL, constant dropped)
"""
from __future__ import annotations

import numpy as np

N_IN, IN_PAD, HID, OUT_PAD = 20, 32, 256, 16
K = [IN_PAD, HID, HID, HID]
N = [HID, HID, HID, OUT_PAD]
S_MIN, S_MAX = -7.0, 5.0


def layout():
    off = 2 * N_IN
    W, b = [], []
    for l in range(4):
        W.append((off, K[l], N[l]))
        off += K[l] * N[l]
        b.append((off, N[l]))
        off += N[l]
    return W, b, off


def unpack(p):
    W_, b_, total = layout()
    assert len(p) == total, (len(p), total)
    p = np.asarray(p, dtype=np.float64)
    mean, std = p[:N_IN], p[N_IN:2 * N_IN]
    Ws = [p[o:o + k * n].reshape(k, n) for o, k, n in W_]
    bs = [p[o:o + n] for o, n in b_]
    return mean, std, Ws, bs


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, X):
    mean, std, Ws, bs = unpack(p)
    x = np.zeros((len(X), IN_PAD))
    x[:, :N_IN] = (np.asarray(X, dtype=np.float64) - mean) / std
    acts, zs = [x], []
    h = x
    for l in range(4):
        z = h @ Ws[l] + bs[l]
        zs.append(z)
        h = silu(z) if l < 3 else z
        acts.append(h)
    return acts, zs


def loss_and_grad(p, X, y):
    """Mean loss and its gradient in the blob layout (normalisation entries get 0)."""
    _, _, Ws, _ = unpack(p)
    acts, zs = forward(p, X)
    out = zs[-1]
    B = len(X)
    y = np.asarray(y, dtype=np.float64)
    mu, s_raw = out[:, 0], out[:, 1]
    s = np.clip(s_raw, S_MIN, S_MAX)
    r = y - mu
    iv = np.exp(-2 * s)
    loss = float(np.mean(s + 0.5 * r * r * iv))
    dz = np.zeros_like(out)
    dz[:, 0] = -r * iv / B
    inside = (s_raw > S_MIN) & (s_raw < S_MAX)
    dz[:, 1] = np.where(inside, (1 - r * r * iv) / B, 0.0)
    W_, b_, total = layout()
    g = np.zeros(total)
    for l in range(3, -1, -1):
        o, k, n = W_[l]
        g[o:o + k * n] = (acts[l].T @ dz).ravel()
        ob, nb = b_[l]
        g[ob:ob + nb] = dz.sum(axis=0)
        if l > 0:
            dz = (dz @ Ws[l].T) * dsilu(zs[l - 1])
    return loss, g


def predict(p, X):
    _, zs = forward(p, X)
    out = zs[-1]
    return out[:, 0], np.exp(np.clip(out[:, 1], S_MIN, S_MAX))
