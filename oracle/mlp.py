"""Per-mode MLP of the learned corrector guess, NumPy FP64 (test
infrastructure only).

The reference has no learned component; this is the CPU oracle for the
product's BF16 MLP kernels (``dnsjax_b200/csrc/learned.cu``,
``dnsjax_b200/csrc/mlp_tc.cu``), for any number of layers:

    h_0 = x,  h_l = relu(h_{l-1} W_l^T + b_l),  y = h_{L-1} W_L^T + b_L,
    L = sum (y - t)^2 / M

with the gradients of L.  The arithmetic is FP64; BF16 rounding is applied
at the points where the GPU path stores BF16 (inputs, weights, hidden
activations, dy and the masked hidden gradients), so the two differ only by
the GPU's FP32 accumulation.  ``finite_difference_check`` checks the
backward pass itself.
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


def _rounder(round_bf16):
    return bf16 if round_bf16 else (lambda a: np.asarray(a, np.float64))


def forward_layers(X, Ws, bs, round_bf16=True):
    """-> (hs, y): hs[0] = the rounded input, hs[l] = hidden layer l as the
    GPU stores it (BF16 when round_bf16), y FP64."""
    r = _rounder(round_bf16)
    hs = [r(X)]
    for W, b in zip(Ws[:-1], bs[:-1]):
        hs.append(r(np.maximum(hs[-1] @ r(W).T + b, 0.0)))
    y = hs[-1] @ r(Ws[-1]).T + bs[-1]
    return hs, y


def loss_and_grads_layers(X, Ws, bs, T, round_bf16=True):
    """Mean-squared-error loss sum((y - t)^2) / M and its gradients
    (lists dWs, dbs), with the GPU path's rounding points."""
    r = _rounder(round_bf16)
    M = X.shape[0]
    hs, y = forward_layers(X, Ws, bs, round_bf16)
    d = y - T
    loss = float(np.sum(d * d) / M)
    dyf = 2.0 * d / M
    cur = r(dyf)
    dWs = [None] * len(Ws)
    dbs = [None] * len(Ws)
    for l in range(len(Ws) - 1, -1, -1):
        dWs[l] = cur.T @ hs[l]
        dbs[l] = dyf.sum(axis=0) if l == len(Ws) - 1 else cur.sum(axis=0)
        if l > 0:
            cur = r((cur @ r(Ws[l])) * (hs[l] > 0))
    return loss, dWs, dbs


def forward(X, W1, b1, W2, b2, round_bf16=True):
    """Two-layer form: -> (h, y)."""
    hs, y = forward_layers(X, [W1, W2], [b1, b2], round_bf16)
    return hs[1], y


def loss_and_grads(X, W1, b1, W2, b2, T, round_bf16=True):
    """Two-layer form: loss and dict(W1, b1, W2, b2) of gradients."""
    loss, dW, db = loss_and_grads_layers(X, [W1, W2], [b1, b2], T, round_bf16)
    return loss, dict(W1=dW[0], b1=db[0], W2=dW[1], b2=db[1])


def adam(w, m, v, g, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One bias-corrected Adam update -> (w, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    w = w - lr * (m / (1 - b1**step)) / (np.sqrt(v / (1 - b2**step)) + eps)
    return w, m, v


def finite_difference_check(seed=0, M=7, K=5, H=6, N=4, eps=1e-6, layers=2) -> float:
    """Largest relative difference between the analytic FP64 gradients (no
    rounding) and central differences of the loss, for a network of
    ``layers`` layers (hidden widths H)."""
    rng = np.random.default_rng(seed)
    sizes = [K] + [H] * (layers - 1) + [N]
    X = rng.standard_normal((M, K))
    T = rng.standard_normal((M, N))
    Ws = [rng.standard_normal((sizes[l + 1], sizes[l])) for l in range(layers)]
    bs = [rng.standard_normal(sizes[l + 1]) * 0.1 for l in range(layers)]
    _, gW, gb = loss_and_grads_layers(X, Ws, bs, T, round_bf16=False)
    worst = 0.0
    for P, G in ((Ws, gW), (bs, gb)):
        for w, g in zip(P, G):
            num = np.zeros_like(w)
            for i in np.ndindex(w.shape):
                old = w[i]
                w[i] = old + eps
                lp, _, _ = loss_and_grads_layers(X, Ws, bs, T, False)
                w[i] = old - eps
                lm, _, _ = loss_and_grads_layers(X, Ws, bs, T, False)
                w[i] = old
                num[i] = (lp - lm) / (2 * eps)
            worst = max(worst, float(np.abs(num - g).max() / max(np.abs(num).max(), 1e-12)))
    return worst
