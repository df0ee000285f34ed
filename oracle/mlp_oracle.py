"""FP64 CPU oracle of the variant selector's network (test infrastructure).

Only the tests use this file, as the checker of the CUDA forward / backward
kernels of sparsep_b200/csrc/mlp.cu.  It restates, in float64 NumPy, the same
network and objective from the same BF16 weights:

  MLP 16 -> 64 -> 64 -> K, ReLU hidden layers; parameters packed as
  W1[64][16], b1[64], W2[64][64], b2[64], W3[K][64], b3[K];
  per sample s over the variants c with t[s, c] > 0:
    p = softmax(z_s) over those c,  r_c = t_c / min t - 1,
    q = softmax(-r / tau) over those c,
    L_s = w_s * (sum_c p_c r_c + lam * sum_c -q_c log p_c),
    w_s = (min t * wscale) ** alpha,
  loss = mean_s L_s (samples with no applicable variant count as 0).

The selector has no counterpart in the reference; nothing here follows a
reference file.
"""
from __future__ import annotations

import numpy as np

F, H = 16, 64


def layout(K: int):
    o = {}
    at = 0
    for name, size in (("W1", H * F), ("b1", H), ("W2", H * H), ("b2", H), ("W3", K * H), ("b3", K)):
        o[name] = (at, at + size)
        at += size
    return o, at


def bf16_bits(w: np.ndarray) -> np.ndarray:
    """float32 -> BF16 bit patterns, round to nearest even (finite inputs)."""
    u = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    return ((u + 0x7FFF + lsb) >> 16).astype(np.uint16)


def bf16_to_f64(b: np.ndarray) -> np.ndarray:
    return (b.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def unpack(w: np.ndarray, K: int):
    o, n = layout(K)
    assert w.size == n
    W1 = w[o["W1"][0]:o["W1"][1]].reshape(H, F)
    W2 = w[o["W2"][0]:o["W2"][1]].reshape(H, H)
    W3 = w[o["W3"][0]:o["W3"][1]].reshape(K, H)
    return W1, w[o["b1"][0]:o["b1"][1]], W2, w[o["b2"][0]:o["b2"][1]], W3, w[o["b3"][0]:o["b3"][1]]


def forward(w: np.ndarray, x: np.ndarray, K: int):
    W1, b1, W2, b2, W3, b3 = unpack(w, K)
    a1 = x @ W1.T + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0.0)
    z = h2 @ W3.T + b3
    return h1, h2, z


def loss_grad(w: np.ndarray, x: np.ndarray, t: np.ndarray, wscale: float, alpha: float = 1.0, lam: float = 0.0,
              tau: float = 0.05):
    """Loss and its gradient w.r.t. the packed weights (all float64)."""
    n, K = t.shape
    w = np.asarray(w, dtype=np.float64)
    x = np.asarray(x, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    W1, b1, W2, b2, W3, b3 = unpack(w, K)
    h1, h2, z = forward(w, x, K)
    mask = t > 0
    anyv = mask.any(axis=1)
    zm = np.where(mask, z, -np.inf)
    zmax = np.where(anyv, zm.max(axis=1), 0.0)
    e = np.where(mask, np.exp(z - zmax[:, None]), 0.0)
    p = e / np.where(anyv, e.sum(axis=1), 1.0)[:, None]
    tb = np.where(anyv, np.where(mask, t, np.inf).min(axis=1), 0.0)
    r = np.where(mask, t / np.where(anyv, tb, 1.0)[:, None] - 1.0, 0.0)
    er = (p * r).sum(axis=1)
    eq = np.where(mask, np.exp(-r / tau), 0.0)
    q = eq / np.where(anyv, eq.sum(axis=1), 1.0)[:, None]
    logp = np.where(mask, z - zmax[:, None] - np.log(np.where(anyv, e.sum(axis=1), 1.0))[:, None], 0.0)
    ce = -(q * logp).sum(axis=1)
    ws = np.where(anyv, (np.where(anyv, tb, 1.0) * wscale) ** alpha, 0.0)
    loss = float((ws * (er + lam * ce)).sum() / n)
    dz = (ws[:, None] * (p * (r - er[:, None]) + lam * (p - q))) / n
    dz = np.where(mask, dz, 0.0)
    dW3 = dz.T @ h2
    db3 = dz.sum(axis=0)
    dh2 = (dz @ W3) * (h2 > 0)
    dW2 = dh2.T @ h1
    db2 = dh2.sum(axis=0)
    dh1 = (dh2 @ W2) * (h1 > 0)
    dW1 = dh1.T @ x
    db1 = dh1.sum(axis=0)
    g = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3])
    return loss, g
