"""CPU float64 restatement of the surrogate network (forward, mean-squared
error, backward) for checking the GPU's BF16 tensor-core kernels.

TEST INFRASTRUCTURE: imported only by tests/, as the checker.

Network: x -> [W_l x + b_l, GELU] x n_hidden -> W_L x + b_L, GELU(z) =
z Phi(z) with the exact normal CDF; loss = mean over batch and outputs of
(pred - y)^2. Parameter layout: layer by layer W [out][in] row-major, then
b [out] (the layout of hc_mlp_get_params).
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np
from scipy.special import erf


def shapes(n_in: int, n_out: int, n_hidden: int, width: int) -> List[Tuple[int, int]]:
    dims = [n_in] + [width] * n_hidden + [n_out]
    return [(dims[i + 1], dims[i]) for i in range(len(dims) - 1)]


def unpack(theta: np.ndarray, shp):
    out, off = [], 0
    for o, i in shp:
        W = theta[off:off + o * i].reshape(o, i)
        off += o * i
        b = theta[off:off + o]
        off += o
        out.append((W, b))
    assert off == theta.size
    return out


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def forward(theta, shp, X):
    layers = unpack(np.asarray(theta, np.float64), shp)
    h = np.asarray(X, np.float64)
    for l, (W, b) in enumerate(layers):
        z = h @ W.T + b
        h = gelu(z) if l + 1 < len(layers) else z
    return h


def loss_and_grad(theta, shp, X, Y):
    layers = unpack(np.asarray(theta, np.float64), shp)
    X = np.asarray(X, np.float64)
    Y = np.asarray(Y, np.float64)
    hs, zs = [X], []
    h = X
    for l, (W, b) in enumerate(layers):
        z = h @ W.T + b
        zs.append(z)
        h = gelu(z) if l + 1 < len(layers) else z
        hs.append(h)
    B, n_out = Y.shape
    d = h - Y
    loss = float(np.mean(d * d))
    g = 2.0 * d / (B * n_out)
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        gW = g.T @ hs[l]
        gb = g.sum(axis=0)
        grads[l] = (gW, gb)
        if l > 0:
            g = (g @ W) * gelu_grad(zs[l - 1])
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, flat
