"""Host-side pieces of the learned warm start (CPU)."""
from __future__ import annotations

import numpy as np


def test_align_removes_rigid_motion():
    from morphoshell_b200 import warmstart as w
    rng = np.random.default_rng(0)
    Q = rng.standard_normal((60, 3))
    a, b, c = 0.7, -0.3, 1.1
    Rz = np.array([[np.cos(a), -np.sin(a), 0], [np.sin(a), np.cos(a), 0], [0, 0, 1]])
    Rx = np.array([[1, 0, 0], [0, np.cos(b), -np.sin(b)], [0, np.sin(b), np.cos(b)]])
    Ry = np.array([[np.cos(c), 0, np.sin(c)], [0, 1, 0], [-np.sin(c), 0, np.cos(c)]])
    P = Q @ (Rz @ Rx @ Ry).T + np.array([1.0, -2.0, 0.5])
    assert np.abs(w.align(P, Q) - Q).max() < 1e-12
    # the mirror image is not a proper rigid motion, shape_distance allows it
    Pm = (Q * np.array([1.0, 1.0, -1.0])) @ Rz.T
    assert w.shape_distance(Q.T.ravel(), Pm.T.ravel()) < 1e-12
    assert w.shape_distance(Q.T.ravel(), (Q + 0.1 * rng.standard_normal(Q.shape)).T.ravel()) > 1e-2


def test_features_continuous_at_centre():
    """Inputs of nodes near the disk centre agree whatever their angle, so
    the predicted displacement has no jump at the defect."""
    from morphoshell_b200 import warmstart as w
    f = w.fields(1, seed=3)[0]
    ang = np.linspace(0.0, 2.0 * np.pi, 16, endpoint=False)
    xy = 1e-6 * np.column_stack([np.cos(ang), np.sin(ang)])
    X = w.node_features(xy, f)
    assert X.shape == (16, w.N_FEATURES)
    assert np.ptp(X, axis=0).max() < 1e-5


def test_fields_deterministic():
    from morphoshell_b200 import warmstart as w
    a, b = w.fields(4, seed=9), w.fields(4, seed=9)
    for x, y in zip(a, b):
        assert np.array_equal(x.a, y.a) and np.array_equal(x.phi, y.phi) and x.lam == y.lam
        assert 0.8 <= x.lam <= 1.2
