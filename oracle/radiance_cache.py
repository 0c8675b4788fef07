"""Numpy restatement of the learned radiance cache's network (test infrastructure).

The cache has no counterpart in the reference renderer; this module is the
oracle its GPU kernels (luz_b200/csrc/cache.cuh) are checked against: the
input encoding, the forward pass with FP16 rounding of inputs, weights and
activations (FP32 accumulation), the relative L2 loss with its clamped,
loss-scaled FP16 output gradient, the backward pass, the weight gradient and
one Adam step. Only tests import it.
"""
from __future__ import annotations

import numpy as np

N_IN, N_ENC, HIDDEN, N_OUT = 10, 128, 64, 16
LAYERS = [(128, 64), (64, 64), (64, 64), (64, 64), (64, 16)]
OFFSETS = [0, 8192, 12288, 16384, 20480]
N_PARAMS = 21504
LOSS_SCALE, GRAD_CLAMP, EPS_REL = 8.0, 2000.0, 0.01
M64 = (1 << 64) - 1


def f16(a):
    return np.asarray(a, np.float32).astype(np.float16).astype(np.float32)


def splitmix64(v: int) -> int:
    v = (v + 0x9E3779B97F4A7C15) & M64
    v = ((v ^ (v >> 30)) * 0xBF58476D1CE4E5B9) & M64
    v = ((v ^ (v >> 27)) * 0x94D049BB133111EB) & M64
    return v ^ (v >> 31)


def init_weights(seed: int) -> np.ndarray:
    """Uniform +-sqrt(6 / fan_in) from splitmix64(seed << 32 ^ index)."""
    w = np.zeros(N_PARAMS, np.float32)
    for (k, n), off in zip(LAYERS, OFFSETS):
        a = np.sqrt(6.0 / k)
        for i in range(k * n):
            u = (splitmix64(((seed << 32) ^ (off + i)) & M64) >> 11) * (1.0 / 9007199254740992.0)
            w[off + i] = np.float32((2.0 * u - 1.0) * a)
    return w


def layers(w: np.ndarray):
    return [w[off:off + k * n].reshape(k, n) for (k, n), off in zip(LAYERS, OFFSETS)]


def encode(x: np.ndarray, exact: bool = False) -> np.ndarray:
    """Column 12 f + 2 k + {0: sin, 1: cos} of (pi 2^k x_f); column 120 is 1."""
    x = np.asarray(x, np.float32)
    e = np.zeros((x.shape[0], N_ENC), np.float64 if exact else np.float32)
    for f in range(N_IN):
        for k in range(6):
            a = (x[:, f] * np.float32(1 << k)).astype(np.float64) * np.pi
            e[:, 12 * f + 2 * k] = np.sin(a)
            e[:, 12 * f + 2 * k + 1] = np.cos(a)
    e[:, 120] = 1.0
    return e if exact else f16(e)


def forward(w: np.ndarray, x: np.ndarray, exact: bool = False):
    """Output (n x 16) and the inputs of every layer: FP16-rounded as on the GPU,
    or in float64 without rounding when exact."""
    r = (lambda a: np.asarray(a, np.float64)) if exact else f16
    W = [r(m) for m in layers(w)]
    acts = [r(encode(x, exact))]
    h = acts[0]
    for l in range(4):
        h = r(np.maximum(h @ W[l], 0.0))
        acts.append(h)
    return h @ W[4], acts


def gradient(w: np.ndarray, x: np.ndarray, t: np.ndarray, exact: bool = False):
    """Mean loss and its gradient with respect to the FP32 weights (flat). exact:
    float64, no rounding and no clamp (for checking the formulas by finite differences)."""
    f16r = (lambda a: np.asarray(a, np.float64)) if exact else f16
    W = [f16r(m) for m in layers(w)]
    y, acts = forward(w, x, exact)
    n = x.shape[0]
    yy = y[:, :3]
    den = yy * yy + (EPS_REL if exact else np.float32(EPS_REL))
    loss = float(np.sum((yy - t) ** 2 / den)) / n
    gy = np.zeros_like(y)
    gy[:, :3] = (2.0 * (yy - t) / den) if exact else np.clip(2.0 * (yy - t) / den, -GRAD_CLAMP, GRAD_CLAMP)
    gy *= LOSS_SCALE
    d = [None] * 5
    d[4] = f16r(gy)
    for l in range(4, 0, -1):
        back = d[l] @ W[l].T
        d[l - 1] = f16r(np.where(acts[l] > 0.0, back, 0.0))
    g = np.zeros(N_PARAMS, np.float64 if exact else np.float32)
    for l, ((k, nn), off) in enumerate(zip(LAYERS, OFFSETS)):
        g[off:off + k * nn] = (acts[l].T @ d[l]).ravel() / (LOSS_SCALE * n)
    return loss, g


def adam(w, m, v, g, step, lr=1e-2, b1=0.9, b2=0.99, eps=1e-8):
    """One Adam step (Kingma & Ba 2015) in place; step counts from 1."""
    m[:] = b1 * m + (1.0 - b1) * g
    v[:] = b2 * v + (1.0 - b2) * g * g
    w[:] -= lr * (m / (1.0 - b1 ** step)) / (np.sqrt(v / (1.0 - b2 ** step)) + eps)
