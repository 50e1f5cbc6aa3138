"""Test oracle of the surrogate network (CPU, numpy FP64). Test infrastructure only: imported by
tests/ as the checker of the GPU kernels, never by the library.

The network has no counterpart in the reference (which has no learned component); this restates
the standard algorithms the GPU path implements:
  * a fully connected network, Z_l = A_{l-1} W_l^T + b_l, A_l = SiLU(Z_l) = Z_l sigmoid(Z_l) for the
    hidden layers, a linear output layer;
  * the mean squared error over rows x outputs and its gradient by back-propagation,
    dL/dZ_l = (dL/dA_l) * SiLU'(Z_l) with SiLU'(z) = s (1 + z (1 - s)), s = sigmoid(z);
  * Adam (Kingma & Ba, ICLR 2015) with bias correction.
With emulate=True the tensors the GPU stores in BF16 (inputs, weights, activations, pre-activations,
output and hidden gradients) are rounded to BF16 (round to nearest even) at the same points, and
everything else is FP64, so the GPU (FP32 accumulation) differs only by accumulation order and the
rare BF16 rounding flip that follows from it.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np


def bf16(x) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32)).view(np.uint32).astype(np.uint64)
    r = ((a + 0x7FFF + ((a >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def shapes(n_in: int, hidden: int, n_hidden: int, n_out: int) -> List[Tuple[int, int]]:
    dims = [n_in] + [hidden] * n_hidden + [n_out]
    return [(dims[i + 1], dims[i]) for i in range(len(dims) - 1)]


def unflatten(p: np.ndarray, n_in, hidden, n_hidden, n_out):
    out, o = [], 0
    for (r, c) in shapes(n_in, hidden, n_hidden, n_out):
        W = p[o:o + r * c].reshape(r, c).astype(np.float64)
        o += r * c
        b = p[o:o + r].astype(np.float64)
        o += r
        out.append((W, b))
    assert o == p.size
    return out


def flatten(layers) -> np.ndarray:
    return np.concatenate([np.concatenate([W.ravel(), b.ravel()]) for W, b in layers])


def init_params(rng: np.random.Generator, n_in, hidden, n_hidden, n_out) -> np.ndarray:
    """He-uniform weights, zero biases."""
    parts = []
    for (r, c) in shapes(n_in, hidden, n_hidden, n_out):
        lim = np.sqrt(6.0 / c)
        parts += [rng.uniform(-lim, lim, r * c), np.zeros(r)]
    return np.concatenate(parts).astype(np.float32)


def _sig(z):
    return 1.0 / (1.0 + np.exp(-z))


def forward(p, x, n_in, hidden, n_hidden, n_out, emulate=True, keep=False):
    q = bf16 if emulate else (lambda v: np.asarray(v, dtype=np.float64))
    layers = unflatten(np.asarray(p, dtype=np.float32), n_in, hidden, n_hidden, n_out)
    A = q(x)
    acts, pre = [A], []
    for i, (W, b) in enumerate(layers):
        Z = A @ q(W).T + b
        if i < len(layers) - 1:
            pre.append(q(Z))
            A = q(Z * _sig(Z))
            acts.append(A)
        else:
            Y = Z
    return (Y, acts, pre) if keep else Y


def gradients(p, x, t, n_in, hidden, n_hidden, n_out, emulate=True, w=None):
    """(flat gradient of the mean squared error, loss); w: optional per-output weights of the
    squared error."""
    q = bf16 if emulate else (lambda v: np.asarray(v, dtype=np.float64))
    layers = unflatten(np.asarray(p, dtype=np.float32), n_in, hidden, n_hidden, n_out)
    Y, acts, pre = forward(p, x, n_in, hidden, n_hidden, n_out, emulate, keep=True)
    rows = x.shape[0]
    D = Y - t
    wv = np.ones(n_out) if w is None else np.asarray(w, dtype=np.float64)
    loss = float(np.mean(wv * D * D))
    dZ = q(wv * D * (2.0 / (rows * n_out)))
    grads = [None] * len(layers)
    for i in range(len(layers) - 1, -1, -1):
        W, _ = layers[i]
        grads[i] = (dZ.T @ acts[i], dZ.sum(axis=0))
        if i > 0:
            dA = dZ @ q(W)
            z = pre[i - 1]
            s = _sig(z)
            dZ = q(dA * s * (1.0 + z * (1.0 - s)))
    return flatten(grads), loss


def adam_step(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (step counts from 1); returns new (p, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    alpha = lr * np.sqrt(1 - b2 ** step) / (1 - b1 ** step)
    return p - alpha * m / (np.sqrt(v) + eps), m, v
