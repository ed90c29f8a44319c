"""CPU oracle of the learned-guess MLP kernels (test infrastructure only).

Restates, in NumPy, what rest_b200/csrc/rijk_mlp.cu computes, so the tests can
check the device kernels' forward values and gradients:

  linear forward   z = x w^T + b (x, w rounded to BF16), y = act(z)
  linear backward  g = dy * act'(z) (FP32), dz = bf16(g); dw = dz^T x; db = sum_rows g; dx = dz w
  masked MSE       loss = sum (mask (y - t))^2 / norm; dy = 2 mask (y - t) / norm
  Adam             the standard bias-corrected update on FP32 masters

BF16 rounding is round-to-nearest-even of the FP32 bit pattern, as
__float2bfloat16_rn does.  Sums are accumulated in float64 here (FP32 on the
device), which sets the comparison tolerance.  REST has no learned guess, so
there is no REST file to cite: the algorithm is the textbook MLP / Adam
(Kingma & Ba, 2015).
"""
from __future__ import annotations

import numpy as np


def bf16_bits(x: np.ndarray) -> np.ndarray:
    """FP32 -> BF16 bit patterns (uint16), round to nearest even (NaN kept quiet)."""
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    rounded = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    nan = np.isnan(np.asarray(x, dtype=np.float32))
    out = rounded.astype(np.uint16)
    out[nan] = 0x7FC0
    return out


def bf16_value(bits: np.ndarray) -> np.ndarray:
    return (np.asarray(bits, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def round_bf16(x: np.ndarray) -> np.ndarray:
    return bf16_value(bf16_bits(x))


def act(kind: int, z: np.ndarray) -> np.ndarray:
    return z / (1.0 + np.exp(-z)) if kind == 1 else z


def act_grad(kind: int, z: np.ndarray) -> np.ndarray:
    if kind != 1:
        return np.ones_like(z)
    s = 1.0 / (1.0 + np.exp(-z))
    return s + z * s * (1.0 - s)


def linear_fwd(x_bits, w_bits, b, kind):
    z = bf16_value(x_bits) @ bf16_value(w_bits).T + (0.0 if b is None else np.asarray(b, dtype=np.float64))
    return z, act(kind, z)


def linear_bwd(x_bits, w_bits, z, dy, kind):
    """db sums the FP32 dz; dw and dx use dz rounded to BF16 (the GEMM operand)."""
    g = (np.asarray(dy, dtype=np.float32) * act_grad(kind, np.asarray(z, np.float64))).astype(np.float32)
    dz = round_bf16(g)
    x, w = bf16_value(x_bits), bf16_value(w_bits)
    return dz.T @ x, g.astype(np.float64).sum(axis=0), dz @ w, dz


def masked_mse(y, t, mask, norm):
    d = (np.asarray(y, np.float64) - t) * (1.0 if mask is None else mask)
    return float(np.sum(d * d) / norm), 2.0 * d / norm


def adam(w, g, m, v, lr, b1, b2, eps, step):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    w = w - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return w, m, v


def network_loss_and_grads(x, ws, bs, target, mask, norm):
    """Whole network in float64 without BF16 rounding (SiLU hidden layers,
    identity output): loss and exact gradients, for finite-difference checks."""
    hs, zs = [np.asarray(x, np.float64)], []
    for i, (w, b) in enumerate(zip(ws, bs)):
        z = hs[-1] @ w.T + b
        zs.append(z)
        hs.append(act(0 if i == len(ws) - 1 else 1, z))
    loss, dy = masked_mse(hs[-1], target, mask, norm)
    grads = [None] * len(ws)
    for i in range(len(ws) - 1, -1, -1):
        dz = dy * act_grad(0 if i == len(ws) - 1 else 1, zs[i])
        grads[i] = (dz.T @ hs[i], dz.sum(axis=0))
        dy = dz @ ws[i]
    return loss, grads
