"""FP64 reference of the learned warm start's MLP (TEST INFRASTRUCTURE: only
the tests and the training report use it as the checker).

27 (padded 32) -> 128 -> 128 -> 128 -> 3 (padded 16), SiLU, parameters in
one flat array in PyTorch Linear layout with the offsets of include/avbd.h.
The reference project has no learned component, so nothing here is pinned
to it: the forward pass is checked against the engine's fused kernel and
the gradient against central differences of this file's own loss.

`bf16=True` rounds weights, inputs and hidden activations to BF16 (round to
nearest even) exactly where the engine's kernels do, keeping FP64 elsewhere.
"""
from __future__ import annotations

import numpy as np

IN, IN_PAD, HID, OUT, OUT_PAD, NPARAMS = 27, 32, 128, 3, 16, 39312
LAYOUT = {"W1": (0, (HID, IN_PAD)), "b1": (4096, (HID,)), "W2": (4224, (HID, HID)), "b2": (20608, (HID,)),
          "W3": (20736, (HID, HID)), "b3": (37120, (HID,)), "W4": (37248, (OUT_PAD, HID)), "b4": (39296, (OUT_PAD,))}


def view(p, name):
    off, shape = LAYOUT[name]
    return p[off:off + int(np.prod(shape))].reshape(shape)


def to_bf16(x):
    """Round FP32/FP64 values to BF16 (nearest, ties to even) and back."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isfinite(f), out, f).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, X, bf16=False):
    """X [n, 32] -> (Y [n, 16], cache)."""
    p = np.asarray(p, dtype=np.float64)
    rw = to_bf16 if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    W = [rw(view(p, f"W{i}")) for i in range(1, 5)]
    b = [view(p, f"b{i}") for i in range(1, 5)]
    h = rw(X)
    cache = {"H0": h, "Z": []}
    for i in range(3):
        z = h @ W[i].T + b[i]
        cache["Z"].append(z)
        h = rw(silu(z))
        cache[f"H{i + 1}"] = h
    y = h @ W[3].T + b[3]
    cache["W"] = W
    return y, cache


def loss_and_grad(p, X, T, bf16=False):
    """Mean over rows and the 3 outputs of w (y - t)^2, w = T[:, 3] the row's
    weight, and its gradient (flat, padding entries zero)."""
    y, c = forward(p, X, bf16)
    n = X.shape[0]
    w = np.asarray(T[:, 3], dtype=np.float64)[:, None]
    e = np.zeros_like(y)
    e[:, :OUT] = y[:, :OUT] - T[:, :OUT]
    loss = float((w * e[:, :OUT] ** 2).sum() / (n * OUT))
    dy = 2.0 * w * e / (n * OUT)
    g = np.zeros(NPARAMS)
    W = c["W"]
    view(g, "W4")[:] = dy.T @ c["H3"]
    view(g, "b4")[:] = dy.sum(0)
    dh = dy @ W[3]
    for i in (2, 1, 0):
        dz = dh * silu_grad(c["Z"][i])
        view(g, f"W{i + 1}")[:] = dz.T @ c[f"H{i}"]
        view(g, f"b{i + 1}")[:] = dz.sum(0)
        dh = dz @ W[i]
    view(g, "W1")[:, IN:] = 0
    view(g, "W4")[OUT:] = 0
    view(g, "b4")[OUT:] = 0
    return loss, g
