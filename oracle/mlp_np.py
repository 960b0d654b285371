"""FP64 numpy restatement of the surrogate MLP (test infrastructure only).

Architecture of the surrogate: 23 inputs (padded to 32) -> 256 -> 256 -> 256
-> 22 outputs (padded to 32), GELU (tanh form, Hendrycks & Gimpel 2016) on
the hidden layers, linear output, loss = mean over the batch of
sum_j w_j (out_j - target_j)^2.  Weights are [out, in] row-major like the
device layout.  Used by the tests to check the forward pass and the
gradients of the device (tcgen05) kernels, and itself checked against
central finite differences.
"""
from __future__ import annotations

import numpy as np

K0 = 0.7978845608028654
K1 = 0.044715


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(K0 * (x + K1 * x ** 3)))


def gelu_grad(x):
    t = np.tanh(K0 * (x + K1 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * K0 * (1.0 + 3.0 * K1 * x * x)


def forward(params, x):
    """params: list of (W [out, in], b [out]); returns (out, cache)."""
    acts = [x]
    pres = []
    h = x
    for li, (W, b) in enumerate(params):
        z = h @ W.T + b
        pres.append(z)
        h = gelu(z) if li < len(params) - 1 else z
        acts.append(h)
    return h, (acts, pres)


def loss_and_grads(params, x, target, w):
    """Weighted MSE: L = mean_b sum_j w_j (out_bj - t_bj)^2; returns (L, grads)."""
    out, (acts, pres) = forward(params, x)
    B = x.shape[0]
    diff = out - target
    L = float(np.sum(w * diff * diff) / B)
    d = 2.0 * w * diff / B
    grads = [None] * len(params)
    for li in range(len(params) - 1, -1, -1):
        W, b = params[li]
        grads[li] = (d.T @ acts[li], d.sum(axis=0))
        if li > 0:
            d = (d @ W) * gelu_grad(pres[li - 1])
    return L, grads


def finite_difference(params, x, target, w, li, which, idx, eps=1e-6):
    """Central difference of the loss w.r.t. one weight (which = 0) or bias (1) entry."""
    def L_at(delta):
        p = [(W.copy(), b.copy()) for W, b in params]
        arr = p[li][which]
        arr[idx] += delta
        return loss_and_grads(p, x, target, w)[0]
    return (L_at(eps) - L_at(-eps)) / (2 * eps)
