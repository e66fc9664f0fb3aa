"""fp32 numpy restatement of the schedule-selector network (test
infrastructure only).

The selector has no counterpart in the reference decoder; this module is the
CPU oracle its CUDA kernels (hpvcd_b200/csrc/selector.cu) are checked
against: the same forward pass, loss and parameter gradients, in float32 on
the bf16-rounded parameters the device forward pass reads.  Only tests/ use
it.
"""
from __future__ import annotations

import numpy as np

F, H = 16, 64


def layout(K: int) -> dict:
    o = {}
    o["w1"] = 0
    o["b1"] = H * F
    o["w2"] = o["b1"] + H
    o["b2"] = o["w2"] + H * H
    o["w3"] = o["b2"] + H
    o["b3"] = o["w3"] + K * H
    o["total"] = o["b3"] + K
    return o


def unpack(p: np.ndarray, K: int):
    L = layout(K)
    p = np.asarray(p)
    W1 = p[L["w1"]:L["b1"]].reshape(H, F)
    b1 = p[L["b1"]:L["w2"]]
    W2 = p[L["w2"]:L["b2"]].reshape(H, H)
    b2 = p[L["b2"]:L["w3"]]
    W3 = p[L["w3"]:L["b3"]].reshape(K, H)
    b3 = p[L["b3"]:L["total"]]
    return W1, b1, W2, b2, W3, b3


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round float32 to the nearest bfloat16 (ties to even), returned as float32."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def forward(p, x, K, dtype=np.float32):
    W1, b1, W2, b2, W3, b3 = (a.astype(dtype) for a in unpack(p, K))
    x = np.asarray(x, dtype)
    h1 = np.maximum(x @ W1.T + b1, 0).astype(dtype)
    h2 = np.maximum(h1 @ W2.T + b2, 0).astype(dtype)
    y = (h2 @ W3.T + b3).astype(dtype)
    return y, h1, h2


def loss(p, x, t, K, dtype=np.float32):
    y, _, _ = forward(p, x, K, dtype)
    return float(np.mean((y - np.asarray(t, dtype)) ** 2))


def loss_and_grad(p, x, t, K, dtype=np.float32):
    """L = mean (y - t)^2 and dL/dp (flat, same layout as p)."""
    W1, b1, W2, b2, W3, b3 = (a.astype(dtype) for a in unpack(p, K))
    x = np.asarray(x, dtype)
    t = np.asarray(t, dtype)
    y, h1, h2 = forward(p, x, K, dtype)
    B = x.shape[0]
    loss = float(np.mean((y - t) ** 2))
    dy = (2.0 * (y - t) / (B * K)).astype(dtype)
    dh2 = (dy @ W3) * (h2 > 0)
    dh1 = (dh2 @ W2) * (h1 > 0)
    g = np.concatenate([(dh1.T @ x).ravel(), dh1.sum(0), (dh2.T @ h1).ravel(), dh2.sum(0),
                        (dy.T @ h2).ravel(), dy.sum(0)]).astype(dtype)
    return loss, g
