"""CPU oracle for the learned queue-order cost model -- TEST INFRASTRUCTURE ONLY.

The reference has no scheduler (it launches one CTA per signal in index order,
kernels.py:1366-1371); the cost model is this build's addition.  This file
restates, in NumPy float64, the 32 per-trace features the feature kernel
computes and the MLP's forward pass, loss gradient and Adam step, so the CUDA
training kernels' gradients can be checked against it.
"""
from __future__ import annotations

import numpy as np

N_FEAT = 32
HIDDEN = 128
N_OUT = 2
N_BANDS = 8
N_SEG = 8
GELU_C = 0.7978845608028654  # sqrt(2/pi)


def trace_features(x: np.ndarray) -> np.ndarray:
    """32 features of one trace (definitions mirrored by the feature kernel)."""
    x = np.asarray(x, dtype=np.float64)
    N = x.shape[0]
    f = np.zeros(N_FEAT)
    if N == 0:
        return f
    e0 = float(np.sum(x * x))
    p0 = e0 / N
    rms = np.sqrt(p0)
    d1 = x[1:] - x[:-1] if N > 1 else np.zeros(0)
    d2 = d1[1:] - d1[:-1] if N > 2 else np.zeros(0)
    e1 = float(np.sum(d1 * d1))
    e2 = float(np.sum(d2 * d2))
    zc = int(np.count_nonzero(x[:-1] * x[1:] < 0.0)) if N > 1 else 0
    if N > 2:
        p = d1[:-1] * d1[1:]
        is_ext = p < 0.0
        nmax = int(np.count_nonzero(is_ext & (d1[:-1] > 0.0)))
        nmin = int(np.count_nonzero(is_ext & (d1[:-1] < 0.0)))
        infl = int(np.count_nonzero(d2[:-1] * d2[1:] < 0.0)) if N > 3 else 0
        ext_idx = np.flatnonzero(is_ext) + 1
    else:
        nmax = nmin = infl = 0
        ext_idx = np.zeros(0, dtype=np.int64)
    f[0] = np.log2(N) / 14.0
    f[1] = N / 16384.0
    f[2] = zc / N
    f[3] = (nmax + nmin) / N
    f[4] = nmax / N
    f[5] = nmin / N
    f[6] = np.log10((e1 + 1e-300) / (e0 + 1e-300)) / 4.0
    f[7] = np.log10((e2 + 1e-300) / (e0 + 1e-300)) / 4.0
    f[8] = infl / N
    # dyadic (Haar) detail energies, levels 1..8
    P = np.concatenate([[0.0], np.cumsum(x)])
    for k in range(N_BANDS):
        w = 1 << k
        npair = N // (2 * w)
        if npair == 0:
            continue
        a = np.arange(npair) * 2 * w
        A = P[a + w] - P[a]
        B = P[a + 2 * w] - P[a + w]
        Dk = float(np.sum((A - B) ** 2)) / (2.0 * w)
        f[9 + k] = Dk / (e0 + 1e-300)
    # extrema density per eighth of the trace
    seg = np.minimum(ext_idx * N_SEG // N, N_SEG - 1) if N else ext_idx
    cnt = np.bincount(seg, minlength=N_SEG)[:N_SEG]
    f[17:25] = cnt * N_SEG / N
    mean = float(np.sum(x)) / N
    q = max(N // 4, 1)
    f[25] = abs(mean) / (rms + 1e-300)
    f[26] = (float(np.sum(x[N - q:])) - float(np.sum(x[:q]))) / q / (rms + 1e-300)
    f[27] = float(np.max(np.abs(x))) / (rms + 1e-300) / 10.0
    f[28] = float(np.sum(x ** 4)) / N / (p0 * p0 + 1e-300) / 10.0
    f[29] = np.count_nonzero(x == 0.0) / N
    f[30] = (np.count_nonzero(d1 == 0.0) / N) if N > 1 else 0.0
    f[31] = np.log10(rms + 1e-300) / 4.0
    return f


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(GELU_C * (z + 0.044715 * z ** 3)))


def gelu_grad(z):
    u = GELU_C * (z + 0.044715 * z ** 3)
    t = np.tanh(u)
    du = GELU_C * (1.0 + 3 * 0.044715 * z ** 2)
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * du


def init_params(seed: int = 0):
    rng = np.random.default_rng(seed)
    def lin(i, o):
        return rng.normal(0.0, np.sqrt(2.0 / i), size=(i, o)), np.zeros(o)
    W1, b1 = lin(N_FEAT, HIDDEN)
    W2, b2 = lin(HIDDEN, HIDDEN)
    W3, b3 = lin(HIDDEN, N_OUT)
    return dict(W1=W1, b1=b1, W2=W2, b2=b2, W3=W3, b3=b3)


def forward(p, X):
    z1 = X @ p["W1"] + p["b1"]
    h1 = gelu(z1)
    z2 = h1 @ p["W2"] + p["b2"]
    h2 = gelu(z2)
    y = h2 @ p["W3"] + p["b3"]
    return y, (X, z1, h1, z2, h2)


def loss_and_grads(p, X, T):
    """Mean squared error over batch and outputs, and its parameter gradients."""
    y, (X, z1, h1, z2, h2) = forward(p, X)
    B = X.shape[0]
    r = y - T
    loss = float(np.mean(r * r))
    dy = 2.0 * r / (B * N_OUT)
    g = {}
    g["W3"] = h2.T @ dy
    g["b3"] = dy.sum(0)
    dz2 = (dy @ p["W3"].T) * gelu_grad(z2)
    g["W2"] = h1.T @ dz2
    g["b2"] = dz2.sum(0)
    dz1 = (dz2 @ p["W2"].T) * gelu_grad(z1)
    g["W1"] = X.T @ dz1
    g["b1"] = dz1.sum(0)
    return loss, g


def adam_step(p, g, m, v, t, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    for k in p:
        m[k] = b1 * m[k] + (1 - b1) * g[k]
        v[k] = b2 * v[k] + (1 - b2) * g[k] * g[k]
        mh = m[k] / (1 - b1 ** t)
        vh = v[k] / (1 - b2 ** t)
        p[k] = p[k] - lr * mh / (np.sqrt(vh) + eps)
    return p, m, v
