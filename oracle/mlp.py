"""Per-mode MLP of the learned corrector guess, NumPy FP64 (test
infrastructure only).

The reference has no learned component; this is the CPU oracle for the
product's BF16 MLP kernels (``dnsjax_b200/csrc/learned.cu``):

    h = relu(x W1^T + b1),   y = h W2^T + b2,   L = sum (y - t)^2 / M

with the gradients of L.  The arithmetic is FP64; BF16 rounding is applied
at the points where the GPU path stores BF16 (inputs, weights, h, dy and
the masked dh), so the two differ only by the GPU's FP32 accumulation.
``finite_difference_check`` checks the backward pass itself.
"""

from __future__ import annotations

import numpy as np


def bf16(a: np.ndarray) -> np.ndarray:
    """Round to bfloat16 (round to nearest even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    nan = np.isnan(f)
    out[nan] = np.nan
    return out


def forward(X, W1, b1, W2, b2, round_bf16=True):
    """-> (h, y): h as the GPU stores it (BF16 when round_bf16), y FP64."""
    r = bf16 if round_bf16 else (lambda a: np.asarray(a, np.float64))
    h = r(np.maximum(r(X) @ r(W1).T + b1, 0.0))
    y = h @ r(W2).T + b2
    return h, y


def loss_and_grads(X, W1, b1, W2, b2, T, round_bf16=True):
    """Mean-squared-error loss sum((y - t)^2) / M and its gradients
    (dW1, db1, dW2, db2), with the GPU path's rounding points."""
    r = bf16 if round_bf16 else (lambda a: np.asarray(a, np.float64))
    M = X.shape[0]
    h, y = forward(X, W1, b1, W2, b2, round_bf16)
    d = y - T
    loss = float(np.sum(d * d) / M)
    dyf = 2.0 * d / M
    dy = r(dyf)
    dW2 = dy.T @ h
    db2 = dyf.sum(axis=0)
    dh = r((dy @ r(W2)) * (h > 0))
    dW1 = dh.T @ r(X)
    db1 = dh.sum(axis=0)
    return loss, dict(W1=dW1, b1=db1, W2=dW2, b2=db2)


def adam(w, m, v, g, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One bias-corrected Adam update -> (w, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    w = w - lr * (m / (1 - b1**step)) / (np.sqrt(v / (1 - b2**step)) + eps)
    return w, m, v


def finite_difference_check(seed=0, M=7, K=5, H=6, N=4, eps=1e-6) -> float:
    """Largest relative difference between the analytic FP64 gradients (no
    rounding) and central differences of the loss."""
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((M, K))
    T = rng.standard_normal((M, N))
    P = dict(W1=rng.standard_normal((H, K)), b1=rng.standard_normal(H) * 0.1,
             W2=rng.standard_normal((N, H)), b2=rng.standard_normal(N) * 0.1)
    _, g = loss_and_grads(X, P["W1"], P["b1"], P["W2"], P["b2"], T, round_bf16=False)
    worst = 0.0
    for k, w in P.items():
        num = np.zeros_like(w)
        for i in np.ndindex(w.shape):
            old = w[i]
            w[i] = old + eps
            lp, _ = loss_and_grads(X, P["W1"], P["b1"], P["W2"], P["b2"], T, False)
            w[i] = old - eps
            lm, _ = loss_and_grads(X, P["W1"], P["b1"], P["W2"], P["b2"], T, False)
            w[i] = old
            num[i] = (lp - lm) / (2 * eps)
        worst = max(worst, float(np.abs(num - g[k]).max() / max(np.abs(num).max(), 1e-12)))
    return worst
