"""The warm-start network on the tensor cores against its CPU oracle -- GPU."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _net(in_dim=22, width=128, hidden=2, out_dim=3, seed=3):
    from morphoshell_b200 import Mlp
    return Mlp(in_dim, width=width, hidden_layers=hidden, out_dim=out_dim, seed=seed)


def _data(n, in_dim=22, out_dim=3, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, in_dim)).astype(np.float32)
    t = np.stack([np.sin(x[:, 0]) * np.cos(x[:, 1]), 0.5 * x[:, 2] * x[:, 3], np.tanh(x[:, 4])][:out_dim], 1)
    return x, t.astype(np.float32)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("n", [128, 300, 1000])
def test_forward_matches_oracle(n):
    from oracle import mlp_ref
    net = _net()
    x, _ = _data(n)
    y = net.forward(x)
    yr = mlp_ref.forward(net.params(), x, 22, 128, 2, 3, bf16_points=True)
    assert _rel(y, yr) < 1e-2
    ye = mlp_ref.forward(net.params(), x, 22, 128, 2, 3, bf16_points=False)
    assert _rel(y, ye) < 5e-2


@pytest.mark.parametrize("width,hidden", [(128, 2), (256, 4)])
def test_gradients_match_oracle(width, hidden):
    """Loss and every layer's weight and bias gradient against the oracle
    with the GPU's bf16 rounding points, and against exact float64."""
    from oracle import mlp_ref
    net = _net(width=width, hidden=hidden)
    x, t = _data(700)
    loss, g = net.loss_grad(x, t)
    lr, gr = mlp_ref.loss_grad(net.params(), x, t, 22, width, hidden, 3, bf16_points=True)
    le, ge = mlp_ref.loss_grad(net.params(), x, t, 22, width, hidden, 3, bf16_points=False)
    assert abs(loss - lr) / lr < 1e-3 and abs(loss - le) / le < 2e-2
    for off, N, K, Np in net.layers():
        w = slice(off, off + N * K)
        b = slice(off + N * K, off + N * K + N)
        assert _rel(g[w], gr[w]) < 2e-2, ("W", off)
        assert _rel(g[b], gr[b]) < 2e-2, ("b", off)
        assert _rel(g[w], ge[w]) < 6e-2
    # padded parameters get no gradient
    off, N, K, Np = net.layers()[-1]
    assert not g[off + N * K + N:off + N * K + Np].any()


def test_training_reduces_loss():
    net = _net(width=128, hidden=2)
    x, t = _data(20000, seed=1)
    net.set_data(x, t)
    losses = net.train(epochs=30, batch=2048, lr=2e-3, seed=0)
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.1 * losses[0], losses
    xv, tv = _data(4000, seed=2)
    yv = net.forward(xv)
    assert float(((yv - tv) ** 2).mean()) < 2 * losses[-1] + 1e-3
