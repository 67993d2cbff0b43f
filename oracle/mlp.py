"""CPU restatement (numpy) of the learned-order cost model, used as the
checker for the CUDA kernels in subgraphmatching_b200/csrc/mlp.cu.

TEST INFRASTRUCTURE ONLY: imported by tests/ (and smoke()); the product never
calls it.  The model has no counterpart in the reference, so this file pins
the kernels' arithmetic, not a reference behaviour: a 64-256-256-1 MLP with
ReLU, weights and hidden activations rounded to bfloat16 (round to nearest
even) exactly where the kernels round them, products accumulated in float
(float64 here, so only summation order separates the two), mean squared
error / 2 loss, and Adam on float32 master weights.

Parameter layout (float32): W1[256][64] b1[256] W2[256][256] b2[256] W3[256] b3[1].
"""
from __future__ import annotations

import numpy as np

IN, HID = 64, 256
SIZES = [("W1", HID * IN), ("b1", HID), ("W2", HID * HID), ("b2", HID), ("W3", HID), ("b3", 1)]
N_PARAMS = sum(n for _, n in SIZES)


def bf16(x) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    nan = ((u & 0x7F800000) == 0x7F800000) & ((u & 0x007FFFFF) != 0)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    r = np.where(nan, ((u >> 16) | 0x40) << 16, r)
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32).reshape(a.shape)


def split(p: np.ndarray) -> dict:
    out, at = {}, 0
    for name, n in SIZES:
        out[name] = p[at:at + n]
        at += n
    out["W1"] = out["W1"].reshape(HID, IN)
    out["W2"] = out["W2"].reshape(HID, HID)
    return out


def forward(p: np.ndarray, x: np.ndarray, rounding: bool = True):
    """Returns (X, H1, H2, Y) as the kernels hold them (X, H1, H2 bfloat16);
    rounding=False keeps everything in float64 (for finite-difference checks)."""
    r = (lambda a: bf16(np.asarray(a, dtype=np.float32)).astype(np.float64)) if rounding else \
        (lambda a: np.asarray(a, dtype=np.float64))
    P = split(np.asarray(p, dtype=np.float64 if not rounding else np.float32))
    X = r(x)
    W1, W2, W3 = (r(P[k]) for k in ("W1", "W2", "W3"))
    H1 = r(np.maximum(X @ W1.T + P["b1"], 0.0))
    H2 = r(np.maximum(H1 @ W2.T + P["b2"], 0.0))
    Y = H2 @ W3 + P["b3"][0]
    return X, H1, H2, Y


def gradients(p: np.ndarray, x: np.ndarray, t: np.ndarray, rounding: bool = True):
    """(grads in the parameter layout, loss) of sum (y - t)^2 / (2n)."""
    P = split(np.asarray(p, dtype=np.float64 if not rounding else np.float32))
    X, H1, H2, Y = forward(p, x, rounding)
    n = len(t)
    d = Y - np.asarray(t, dtype=np.float64)
    loss = float((d * d).sum() / (2 * n))
    dY = d / n
    W2, W3 = ((bf16(P[k]).astype(np.float64) if rounding else np.asarray(P[k], dtype=np.float64))
              for k in ("W2", "W3"))
    gW3 = dY @ H2
    gb3 = np.array([dY.sum()])
    dH2 = np.outer(dY, W3) * (H2 > 0)
    gW2 = dH2.T @ H1
    gb2 = dH2.sum(0)
    dH1 = (dH2 @ W2) * (H1 > 0)
    gW1 = dH1.T @ X
    gb1 = dH1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, gb3])
    return (g.astype(np.float32) if rounding else g), loss


def adam(p, g, m, v, step: int, lr: float, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (bias-corrected) on float32 master weights."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    c1, c2 = 1 - b1 ** step, 1 - b2 ** step
    p = p - lr * (m / c1) / (np.sqrt(v / c2) + eps)
    return p.astype(np.float32), m.astype(np.float32), v.astype(np.float32)
