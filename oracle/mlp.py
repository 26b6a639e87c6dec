"""TEST INFRASTRUCTURE ONLY: float64 numpy restatement of the warm-start network's forward
and backward passes (33 -> 256 -> 256 -> K, exact-erf GELU, softmax(f(x) + prior),
mean cross-entropy against soft targets), used to check the CUDA kernels' outputs and
gradients. The weights given are the BF16-rounded values the kernels read, and every
matrix product rounds its two inputs to BF16 first, as the kernels' tensor-core GEMMs do
(the products and sums stay float64 here). (The network is this library's own component;
the reference has none.)"""
from __future__ import annotations

import math

import numpy as np

_erf = np.vectorize(math.erf)


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    cdf = 0.5 * (1.0 + _erf(x / math.sqrt(2.0)))
    return cdf + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def bf(x):
    """x rounded to BF16 (round to nearest even, through float32), as float64."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(X, prior, W1, b1, W2, b2, W3, b3):
    h1p = bf(X) @ bf(W1).T + b1
    h1 = gelu(h1p)
    h2p = bf(h1) @ bf(W2).T + b2
    h2 = gelu(h2p)
    z = bf(h2) @ bf(W3).T + b3 + prior
    z = z - z.max(1, keepdims=True)
    p = np.exp(z)
    p /= p.sum(1, keepdims=True)
    return dict(h1p=h1p, h1=h1, h2p=h2p, h2=h2, z=z, p=p)


def backward(X, T, W2, W3, cache):
    B = X.shape[0]
    p = cache["p"]
    loss = float(-(T * np.log(np.maximum(p, 1e-300))).sum() / B)
    dz = (p - T) / B
    g = {"W3": bf(dz).T @ bf(cache["h2"]), "b3": dz.sum(0)}
    d2 = (bf(dz) @ bf(W3)) * gelu_grad(cache["h2p"])
    g["W2"], g["b2"] = bf(d2).T @ bf(cache["h1"]), d2.sum(0)
    d1 = (bf(d2) @ bf(W2)) * gelu_grad(cache["h1p"])
    g["W1"], g["b1"] = bf(d1).T @ bf(X), d1.sum(0)
    return loss, g
