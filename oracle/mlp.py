"""CPU restatement of the pivot MLP (test infrastructure only).

The learned pivot has no reference counterpart; this file is the checker for
the library's hand-written CUDA kernels (kaspan_b200/csrc/mlp.cu): the same
eight vertex features, the same BF16 rounding of the weights (round to
nearest even), and forward pass, mean binary cross-entropy and its gradient
in float64.  Only tests/ import it.
"""
from __future__ import annotations

import numpy as np

IN, H = 8, 32
O_W1 = 0
O_B1 = O_W1 + H * IN
O_W2 = O_B1 + H
O_B2 = O_W2 + H * H
O_W3 = O_B2 + H
O_B3 = O_W3 + H
NPARAM = O_B3 + 1
SAMPLE = 64


def bf16(x: np.ndarray) -> np.ndarray:
    """float32 -> the nearest bfloat16 (ties to even), returned as float32."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)


def unpack(params: np.ndarray):
    p = bf16(params).astype(np.float64)
    return (p[O_W1:O_B1].reshape(H, IN), p[O_B1:O_W2], p[O_W2:O_B2].reshape(H, H), p[O_B2:O_W3], p[O_W3:O_B3], p[O_B3])


def features(fwh, fwc, bwh, bwc, vertices) -> np.ndarray:
    """The eight features of each vertex (kaspan_b200/csrc/mlp.cuh header)."""
    fwh = fwh.astype(np.int64)
    bwh = bwh.astype(np.int64)
    out_deg = np.diff(fwh)
    in_deg = np.diff(bwh)
    F = np.zeros((len(vertices), IN), np.float64)
    lg = lambda x: np.log2(1.0 + x) / 16.0  # noqa: E731
    live = (out_deg > 0) & (in_deg > 0)  # survives trim round 1 (trim_1_local.hpp:12-46)
    for r, v in enumerate(vertices):
        on = fwc[fwh[v]: fwh[v] + min(out_deg[v], SAMPLE)].astype(np.int64)
        inn = bwc[bwh[v]: bwh[v] + min(in_deg[v], SAMPLE)].astype(np.int64)
        F[r, 0] = lg(out_deg[v])
        F[r, 1] = lg(in_deg[v])
        F[r, 2] = lg(out_deg[on].mean()) if len(on) else 0.0
        F[r, 3] = lg(in_deg[inn].mean()) if len(inn) else 0.0
        F[r, 4] = live[on].mean() if len(on) else 0.0
        F[r, 5] = live[inn].mean() if len(inn) else 0.0
        # the trim round that removes v, judged from its samples: 1 (a
        # degree is 0), 2 (no sampled out- or in-neighbour survives round 1),
        # later or never
        if not len(on) or not len(inn):
            F[r, 6] = 0.0
        elif not live[on].any() or not live[inn].any():
            F[r, 6] = 0.5
        else:
            F[r, 6] = 1.0
        F[r, 7] = lg(out_deg[inn].mean()) if len(inn) else 0.0
    return F


def forward(params: np.ndarray, x: np.ndarray):
    W1, b1, W2, b2, w3, b3 = unpack(params)
    a1 = x @ W1.T + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0.0)
    z = h2 @ w3 + b3
    return z, (x, a1, h1, a2, h2)


def loss_and_grad(params: np.ndarray, x: np.ndarray, y: np.ndarray):
    """Mean BCE of sigmoid(z) vs y and its gradient w.r.t. the parameters
    (through the BF16 rounding as the identity)."""
    W1, b1, W2, b2, w3, b3 = unpack(params)
    z, (x, a1, h1, a2, h2) = forward(params, x)
    n = len(y)
    loss = np.mean(np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z))))
    dz = (1.0 / (1.0 + np.exp(-z)) - y) / n
    g = np.zeros(NPARAM)
    g[O_B3] = dz.sum()
    g[O_W3:O_B3] = h2.T @ dz
    d2 = (dz[:, None] * w3[None, :]) * (a2 > 0)
    g[O_B2:O_W3] = d2.sum(0)
    g[O_W2:O_B2] = (d2.T @ h1).reshape(-1)
    d1 = (d2 @ W2) * (a1 > 0)
    g[O_B1:O_W2] = d1.sum(0)
    g[O_W1:O_B1] = (d1.T @ x).reshape(-1)
    return loss, g
