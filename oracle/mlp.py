"""ORACLE — test infrastructure only.

NumPy restatement (float64) of the selector network of libvpm_fmm.so, used by
tests/ as the checker of the GPU forward and backward kernels; never part of
the product. Layout and definitions follow include/vpm_fmm.h: layers
228 -> 64 -> 64 -> 64 -> 70, parameters per layer W [out x in] then b [out],
GELU 0.5 z (1 + erf(z / sqrt 2)) after the hidden layers, loss = mean over
all B x 70 entries of (mask (yhat - y))^2.
"""
from __future__ import annotations

import math

import numpy as np

DIMS = (228, 64, 64, 64, 70)

_erf = np.vectorize(math.erf)


def param_count() -> int:
    return sum(DIMS[l + 1] * DIMS[l] + DIMS[l + 1] for l in range(len(DIMS) - 1))


def unpack(params):
    out, o = [], 0
    for l in range(len(DIMS) - 1):
        i, n = DIMS[l], DIMS[l + 1]
        W = params[o:o + n * i].reshape(n, i)
        o += n * i
        b = params[o:o + n]
        o += n
        out.append((W, b))
    return out


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    cdf = 0.5 * (1.0 + _erf(z / math.sqrt(2.0)))
    pdf = np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)
    return cdf + z * pdf


def forward(params, X):
    """Outputs and the per-layer (input, pre-activation) cache."""
    A = np.asarray(X, dtype=np.float64)
    cache = []
    layers = unpack(np.asarray(params, dtype=np.float64))
    for l, (W, b) in enumerate(layers):
        Z = A @ W.T + b
        cache.append((A, Z))
        A = gelu(Z) if l + 1 < len(layers) else Z
    return A, cache


def loss_and_grads(params, X, Y, mask=None):
    params = np.asarray(params, dtype=np.float64)
    Yh, cache = forward(params, X)
    M = np.ones_like(Yh) if mask is None else np.asarray(mask, dtype=np.float64)
    n = Yh.size
    d = (Yh - np.asarray(Y, dtype=np.float64)) * M
    loss = float(np.sum(d * d) / n)
    dA = 2.0 * d / n
    layers = unpack(params)
    grads = []
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        A_in, Z = cache[l]
        dZ = dA * gelu_grad(Z) if l + 1 < len(layers) else dA
        grads.append((dZ.T @ A_in, dZ.sum(axis=0)))
        dA = dZ @ W
    flat = []
    for dW, db in reversed(grads):
        flat.append(dW.ravel())
        flat.append(db)
    return loss, np.concatenate(flat)
