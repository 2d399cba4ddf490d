"""Float64 CPU restatement of the traversal-variant selector network
(TEST INFRASTRUCTURE ONLY: the checker for the library's hand-written MLP
kernels; nothing in the library calls it).

Network: 10 -> 32 -> 32 -> 4, ReLU after the two hidden layers, linear
output = predicted log2 time (microseconds) of each of the four traversal
variants.  Parameters are packed in this order (float32 in the library):
    W1[32][10], b1[32], W2[32][32], b2[32], W3[4][32], b3[4]
Loss: masked mean squared error over (sample, variant) pairs with mask 1,
    L = sum(mask * (out - y)^2) / max(1, sum(mask)).
"""
from __future__ import annotations

import numpy as np

D_IN, H1, H2, D_OUT = 10, 32, 32, 4
SHAPES = [(H1, D_IN), (H1,), (H2, H1), (H2,), (D_OUT, H2), (D_OUT,)]
N_PARAMS = sum(int(np.prod(s)) for s in SHAPES)


def unpack(p: np.ndarray):
    out, k = [], 0
    for s in SHAPES:
        c = int(np.prod(s))
        out.append(np.asarray(p[k:k + c], dtype=np.float64).reshape(s))
        k += c
    return out


def pack(ws) -> np.ndarray:
    return np.concatenate([np.asarray(w, dtype=np.float64).ravel() for w in ws])


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    f = np.asarray(x, dtype=np.float32).copy()
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(p: np.ndarray, X: np.ndarray):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    z1 = X @ W1.T + b1
    a1 = np.maximum(z1, 0)
    z2 = a1 @ W2.T + b2
    a2 = np.maximum(z2, 0)
    out = a2 @ W3.T + b3
    return out, (X, z1, a1, z2, a2)


def loss_and_grad(p: np.ndarray, X: np.ndarray, Y: np.ndarray, M: np.ndarray):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    out, (X, z1, a1, z2, a2) = forward(p, X)
    M = np.asarray(M, dtype=np.float64)
    cnt = max(1.0, M.sum())
    r = (out - np.asarray(Y, dtype=np.float64)) * M
    loss = float((r * r).sum() / cnt)
    g_out = 2.0 * r / cnt
    gW3 = g_out.T @ a2
    gb3 = g_out.sum(0)
    g_a2 = g_out @ W3
    g_z2 = g_a2 * (z2 > 0)
    gW2 = g_z2.T @ a1
    gb2 = g_z2.sum(0)
    g_a1 = g_z2 @ W2
    g_z1 = g_a1 * (z1 > 0)
    gW1 = g_z1.T @ X
    gb1 = g_z1.sum(0)
    return loss, pack([gW1, gb1, gW2, gb2, gW3, gb3])


def init_params(seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    ws = []
    for s in SHAPES:
        if len(s) == 2:
            ws.append(rng.normal(0, np.sqrt(2.0 / s[1]), size=s))
        else:
            ws.append(np.zeros(s))
    return pack(ws).astype(np.float32)
