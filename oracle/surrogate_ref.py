# SPDX-License-Identifier: 0BSD
"""Test infrastructure: a plain numpy FP64 restatement of the learned
super-stepper (5 layers of 3x3 convolutions, zero padding, GELU) with its
backward pass and AdamW, the checker for the tensor-core kernels and the
training step.  Not used by the product path.

Layouts follow the library's: activations NHWC; weights W[c_out, tap, c_in]
with tap = 3 * (dy + 1) + (dx + 1), packed [c_out][9 * c_in] (tap-major).
"""
from __future__ import annotations

import math

import numpy as np

TAPS = [(t // 3 - 1, t % 3 - 1) for t in range(9)]
CH = (4, 32, 32, 32, 32, 1)          # channels of the 5 layers' inputs/outputs


def conv3x3(x: np.ndarray, w: np.ndarray, b: np.ndarray | None = None) -> np.ndarray:
    """x [B, H, W, Cin], w [Cout, 9, Cin] -> [B, H, W, Cout]."""
    B, H, W, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    out = np.zeros((B, H, W, w.shape[0]))
    for t, (dy, dx) in enumerate(TAPS):
        out += xp[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W, :] @ w[:, t, :].T
    if b is not None:
        out += b
    return out


def conv3x3_input_grad(g: np.ndarray, w: np.ndarray) -> np.ndarray:
    """Gradient w.r.t. the input of conv3x3 for upstream gradient g [B,H,W,Cout]."""
    return conv3x3(g, flip_transpose(w))


def conv3x3_weight_grad(x: np.ndarray, g: np.ndarray):
    """(dW [Cout, 9, Cin], db [Cout]) for input x and upstream gradient g."""
    B, H, W, C = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    dw = np.zeros((g.shape[-1], 9, C))
    gf = g.reshape(-1, g.shape[-1])
    for t, (dy, dx) in enumerate(TAPS):
        dw[:, t, :] = gf.T @ xp[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W, :].reshape(-1, C)
    return dw, gf.sum(axis=0)


def flip_transpose(w: np.ndarray) -> np.ndarray:
    """W'[ci, t, co] = W[co, 8 - t, ci]: the input-gradient weights."""
    return np.ascontiguousarray(w[:, ::-1, :].transpose(2, 1, 0))


def pack(w: np.ndarray, n_pad: int | None = None, k_pad: int | None = None) -> np.ndarray:
    """[Cout, 9, Cin] -> [N][K] with K = 9 Cin (zero-padded to k_pad), N to n_pad."""
    co, _, ci = w.shape
    p = w.reshape(co, 9 * ci)
    K = max(9 * ci, k_pad or 0)
    N = max(co, n_pad or 0)
    out = np.zeros((N, K))
    out[:co, :9 * ci] = p
    return out


GELU_C, GELU_A = math.sqrt(2.0 / math.pi), 0.044715


def gelu(x):
    """GELU, tanh form (Hendrycks and Gimpel 2016), as the kernels use it."""
    return 0.5 * x * (1.0 + np.tanh(GELU_C * (x + GELU_A * x ** 3)))


def gelu_grad(x):
    t = np.tanh(GELU_C * (x + GELU_A * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * GELU_C * (1.0 + 3.0 * GELU_A * x * x)


def init_params(seed: int = 0):
    """He-style initial weights (fp64): list of (W [Cout, 9, Cin], b [Cout])."""
    rng = np.random.default_rng(seed)
    ps = []
    for li in range(5):
        ci, co = CH[li], CH[li + 1]
        std = math.sqrt(2.0 / (9 * ci)) if li < 4 else 0.1 * math.sqrt(1.0 / (9 * ci))
        ps.append((rng.normal(0.0, std, (co, 9, ci)), np.zeros(co)))
    return ps


def forward(params, x):
    """Returns (y [B,H,W], cache) with cache = inputs and pre-activations."""
    acts, pres = [x], []
    h = x
    for li, (w, b) in enumerate(params):
        pre = conv3x3(h, w, b)
        pres.append(pre)
        h = gelu(pre) if li < 4 else pre
        acts.append(h)
    return h[..., 0], (acts, pres)


def loss_and_grads(params, x, target):
    """Mean squared error over pixels and its gradients (list of (dW, db))."""
    y, (acts, pres) = forward(params, x)
    P = y.size
    r = y - target
    loss = float(np.sum(r * r) / P)
    g = (2.0 / P * r)[..., None]                 # d loss / d pre5
    grads = [None] * 5
    for li in range(4, -1, -1):
        dw, db = conv3x3_weight_grad(acts[li], g)
        grads[li] = (dw, db)
        if li > 0:
            g = conv3x3_input_grad(g, params[li][0]) * gelu_grad(pres[li - 1])
    return loss, grads


def adamw(p, g, m, v, step, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, wd=0.01):
    """One AdamW update (decoupled weight decay); returns (p, m, v)."""
    m = beta1 * m + (1 - beta1) * g
    v = beta2 * v + (1 - beta2) * g * g
    mh = m / (1 - beta1 ** step)
    vh = v / (1 - beta2 ** step)
    p = p - lr * (mh / (np.sqrt(vh) + eps) + wd * p)
    return p, m, v
