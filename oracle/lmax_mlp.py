"""Oracle (test infrastructure only): FP64 numpy restatement of the learned
cutoff network -- forward, mean-squared loss and backward -- for checking
the GPU kernels' gradients.  Weights are rounded to bf16 exactly as the GPU
kernels round them (round to nearest even); biases and the standardisation
stay FP32.  Only tests may import this module.

Parameter block layout (float32, 34713 entries):
  x_mean[11] x_std[11] y_mean y_std | W1[128][11] b1[128] | W2[128][128]
  b2[128] | W3[128][128] b3[128] | W4[128] b4
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

NF, H = 11, 128
OFF_XM, OFF_XS, OFF_YM, OFF_YS = 0, NF, 2 * NF, 2 * NF + 1
OFF_W1 = 2 * NF + 2
OFF_B1 = OFF_W1 + H * NF
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H * H
OFF_W4 = OFF_B3 + H
OFF_B4 = OFF_W4 + H
NPARAM = OFF_B4 + 1


def bf16(x: np.ndarray) -> np.ndarray:
    """float32 -> bf16 (round to nearest even) -> float64."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def dgelu(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def unpack(P):
    P = np.asarray(P)
    W1 = bf16(P[OFF_W1:OFF_B1]).reshape(H, NF)
    W2 = bf16(P[OFF_W2:OFF_B2]).reshape(H, H)
    W3 = bf16(P[OFF_W3:OFF_B3]).reshape(H, H)
    W4 = bf16(P[OFF_W4:OFF_B4])
    b = [P[OFF_B1:OFF_W2].astype(np.float64), P[OFF_B2:OFF_W3].astype(np.float64),
         P[OFF_B3:OFF_W4].astype(np.float64), float(P[OFF_B4])]
    return (W1, W2, W3, W4), b


def loss_and_grad(P, X, T):
    """MSE of the standardised output and its gradient (float64 arrays).
    P as the GPU holds it (float32); a float64 P is used as given."""
    P = np.asarray(P)
    (W1, W2, W3, W4), (b1, b2, b3, b4) = unpack(P)
    xm, xs = P[OFF_XM:OFF_XS].astype(np.float64), P[OFF_XS:OFF_YM].astype(np.float64)
    ym, ys = float(P[OFF_YM]), float(P[OFF_YS])
    Xn = (np.asarray(X, np.float64) - xm) / xs
    t = (np.asarray(T, np.float64) - ym) / ys
    n = len(t)
    z1 = Xn @ W1.T + b1
    a1 = gelu(z1)
    z2 = a1 @ W2.T + b2
    a2 = gelu(z2)
    z3 = a2 @ W3.T + b3
    a3 = gelu(z3)
    y = a3 @ W4 + b4
    d = y - t
    loss = float(np.mean(d * d))
    dy = 2.0 * d / n
    G = np.zeros(NPARAM)
    G[OFF_W4:OFF_B4] = dy @ a3
    G[OFF_B4] = dy.sum()
    dz3 = np.outer(dy, W4) * dgelu(z3)
    G[OFF_W3:OFF_B3] = (dz3.T @ a2).reshape(-1)
    G[OFF_B3:OFF_W4] = dz3.sum(0)
    dz2 = (dz3 @ W3) * dgelu(z2)
    G[OFF_W2:OFF_B2] = (dz2.T @ a1).reshape(-1)
    G[OFF_B2:OFF_W3] = dz2.sum(0)
    dz1 = (dz2 @ W2) * dgelu(z1)
    G[OFF_W1:OFF_B1] = (dz1.T @ Xn).reshape(-1)
    G[OFF_B1:OFF_W2] = dz1.sum(0)
    return loss, G, y * ys + ym


def init(X, T, seed=0):
    """Same standardisation rule as the library; weights from numpy (only
    the layout matters for the checks)."""
    X = np.asarray(X, np.float64)
    T = np.asarray(T, np.float64)
    P = np.zeros(NPARAM, np.float32)
    P[OFF_XM:OFF_XS] = X.mean(0)
    sd = X.std(0)
    P[OFF_XS:OFF_YM] = np.where(sd > 1e-6, sd, 1.0)
    P[OFF_YM] = T.mean()
    P[OFF_YS] = T.std() if T.std() > 1e-6 else 1.0
    rng = np.random.default_rng(seed)
    P[OFF_W1:OFF_B1] = rng.normal(0, np.sqrt(2 / NF), H * NF)
    P[OFF_W2:OFF_B2] = rng.normal(0, np.sqrt(2 / H), H * H)
    P[OFF_W3:OFF_B3] = rng.normal(0, np.sqrt(2 / H), H * H)
    P[OFF_W4:OFF_B4] = rng.normal(0, np.sqrt(2 / H), H)
    P[OFF_B1:OFF_W2] = rng.normal(0, 0.1, H)
    P[OFF_B2:OFF_W3] = rng.normal(0, 0.1, H)
    P[OFF_B3:OFF_W4] = rng.normal(0, 0.1, H)
    return P
