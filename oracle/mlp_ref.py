"""CPU oracle of the warm-start network -- TEST INFRASTRUCTURE ONLY.

A numpy restatement of the SiLU MLP that ms_mlp_* trains on the tensor
cores: same parameter layout (per layer W [N][K] row-major then the padded
bias [Np]), same loss (mean squared error over rows and outputs), and, with
``bf16=True``, the same rounding points as the GPU path (inputs, weights,
pre-activations Z, activations H, and the backward dZ rounded to bfloat16;
products accumulated in double here, in FP32 on the GPU).  With
``bf16=False`` it is the exact-arithmetic network in float64.  The network
has no counterpart in the reference (it replaces the ansatz of
move_nodes_to_ansatz_positions.cpp:31-38 as a start state).
"""
from __future__ import annotations

import numpy as np


def bf16(a: np.ndarray) -> np.ndarray:
    """Round to bfloat16 (nearest, ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def layers(in_dim: int, width: int, hidden: int, out_dim: int):
    in_pad = (in_dim + 15) // 16 * 16
    out, off = [], 0
    nl = hidden + 1
    for l in range(nl):
        K = in_pad if l == 0 else width
        N = out_dim if l == nl - 1 else width
        Np = 16 if l == nl - 1 else width
        out.append((off, N, K, Np))
        off += N * K + Np
    return out, in_pad


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def loss_grad(params, x, t, in_dim, width, hidden, out_dim, bf16_points=True):
    """(loss, gradient vector) of one batch."""
    q = bf16 if bf16_points else (lambda a: np.asarray(a, dtype=np.float64))
    lay, in_pad = layers(in_dim, width, hidden, out_dim)
    p = np.asarray(params, dtype=np.float64)
    n = x.shape[0]
    X = np.zeros((n, in_pad))
    X[:, :in_dim] = x
    X = q(X)
    Ws, bs = [], []
    for off, N, K, Np in lay:
        Ws.append(q(p[off:off + N * K].reshape(N, K)))
        bs.append(p[off + N * K:off + N * K + N])
    Hs, Zs = [X], []
    h = X
    for l, (W, b) in enumerate(zip(Ws, bs)):
        z = h @ W.T + b
        if l < len(Ws) - 1:
            z = q(z)
            Zs.append(z)
            h = q(_silu(z))
            Hs.append(h)
        else:
            y = z.astype(np.float32).astype(np.float64) if bf16_points else z
    d = y - t
    loss = float((d * d).sum() / (n * out_dim))
    dz = q(2.0 * d / (n * out_dim))
    g = np.zeros_like(p)
    for l in range(len(Ws) - 1, -1, -1):
        off, N, K, Np = lay[l]
        g[off:off + N * K] = (dz.T @ Hs[l]).ravel()
        g[off + N * K:off + N * K + N] = dz.sum(0)
        if l == 0:
            break
        dh = dz @ Ws[l]
        dz = q(dh * _dsilu(Zs[l - 1]))
    return loss, g


def forward(params, x, in_dim, width, hidden, out_dim, bf16_points=True):
    lay, in_pad = layers(in_dim, width, hidden, out_dim)
    q = bf16 if bf16_points else (lambda a: np.asarray(a, dtype=np.float64))
    p = np.asarray(params, dtype=np.float64)
    X = np.zeros((x.shape[0], in_pad))
    X[:, :in_dim] = x
    h = q(X)
    for l, (off, N, K, Np) in enumerate(lay):
        W = q(p[off:off + N * K].reshape(N, K))
        z = h @ W.T + p[off + N * K:off + N * K + N]
        if l < len(lay) - 1:
            h = q(_silu(q(z)))
    return z
