"""Oracle: forward and backward of the field-surrogate MLP (NumPy, float64),
with BF16 rounding applied where the CUDA kernels store BF16 (weights of the
tensor-core layers, hidden activations, backpropagated deltas) so gradients
can be compared tightly.  Test infrastructure only -- see oracle/__init__.py.

Network: x (2) -> 128 -> 128 -> 128 -> 128 -> y (2), SiLU after every hidden
layer; loss = mean over the batch of |y - t|^2.
"""

import numpy as np


def bf16(a):
    """Round float64/float32 values to bfloat16 (round to nearest even) and back."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward_backward(p, x, t):
    """p: dict W1 [128,2], b1, W2..W4 [128,128], b2..b4, W5 [2,128], b5.
    Returns (loss, grads dict, y)."""
    B = len(x)
    W = {k: np.asarray(v, dtype=np.float64) for k, v in p.items()}
    W1, W5 = bf16(W["W1"]), bf16(W["W5"])
    Wl = {l: bf16(W[f"W{l}"]) for l in (2, 3, 4)}
    z = {1: x @ W1.T + W["b1"]}
    h = {1: bf16(silu(z[1]))}
    for l in (2, 3, 4):
        z[l] = h[l - 1] @ Wl[l].T + W[f"b{l}"]
        h[l] = bf16(silu(z[l]))
    y = h[4] @ W5.T + W["b5"]
    e = y - t
    loss = np.sum(e * e) / B
    dy = 2.0 * e / B
    g = {"W5": dy.T @ h[4], "b5": dy.sum(0)}
    d = bf16((dy @ W5) * dsilu(z[4]))
    for l in (4, 3, 2):
        g[f"W{l}"] = d.T @ h[l - 1]
        g[f"b{l}"] = d.sum(0)
        d = bf16((d @ Wl[l]) * dsilu(z[l - 1]))
    g["W1"] = d.T @ x
    g["b1"] = d.sum(0)
    return loss, g, y
