"""The network oracle's gradient against central finite differences (CPU)."""
from __future__ import annotations

import numpy as np


def test_oracle_gradient_finite_differences():
    from oracle import mlp_ref
    rng = np.random.default_rng(0)
    in_dim, width, hidden, out_dim = 5, 16, 2, 3
    lay, in_pad = mlp_ref.layers(in_dim, width, hidden, out_dim)
    n_par = lay[-1][0] + lay[-1][1] * lay[-1][2] + lay[-1][3]
    p = rng.standard_normal(n_par) * 0.5
    for off, N, K, Np in lay:  # padded bias entries and padded input columns stay zero
        p[off + N * K + N:off + N * K + Np] = 0.0
        if off == 0:
            w = p[off:off + N * K].reshape(N, K)
            w[:, in_dim:] = 0.0
    x = rng.standard_normal((9, in_dim))
    t = rng.standard_normal((9, out_dim))
    loss, g = mlp_ref.loss_grad(p, x, t, in_dim, width, hidden, out_dim, bf16_points=False)
    idx = rng.choice(n_par, 60, replace=False)
    for i in idx:
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp, _ = mlp_ref.loss_grad(pp, x, t, in_dim, width, hidden, out_dim, bf16_points=False)
        lm, _ = mlp_ref.loss_grad(pm, x, t, in_dim, width, hidden, out_dim, bf16_points=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_bf16_rounding():
    from oracle import mlp_ref
    a = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -3.14159, 1e-30, 65504.0])
    r = mlp_ref.bf16(a)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == 1.0 + 2 ** -7
    assert abs(r[3] + 3.140625) < 1e-12
    assert np.all(np.abs(r - a) <= np.abs(a) * 2 ** -8)
