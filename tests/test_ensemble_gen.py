"""The batched-ensemble workload generator (CPU)."""
from __future__ import annotations

import math

import numpy as np


def test_ensemble_params_distribution():
    from morphoshell_b200 import meshgen
    ps = [meshgen.ensemble_params(k, seed=7) for k in range(256)]
    sp = np.array([p["spacing"] for p in ps])
    assert sp.min() >= 0.004 and sp.max() <= 0.02
    # log-uniform: the median is near the geometric mean of the range
    assert abs(math.log(np.median(sp)) - 0.5 * (math.log(0.004) + math.log(0.02))) < 0.25
    lam = np.array([p["lam_final"] for p in ps])
    assert lam.min() >= 0.8 and lam.max() <= 1.2 and (lam < 1).any() and (lam > 1).any()
    h = np.array([p["thickness"] for p in ps])
    assert h.min() >= 0.005 and h.max() <= 0.02
    assert {p["charge"] for p in ps} == {1.0, -1.0, 0.5}
    assert meshgen.ensemble_params(5, seed=7) == ps[5]
    assert meshgen.ensemble_params(5, seed=8) != ps[5]


def test_ensemble_member_field(tmp_path):
    """The director of member k is charge * theta at triangle centroids."""
    from morphoshell_b200 import meshgen
    mesh, info, bbar, over, p = meshgen.ensemble_member(3, seed=7, spacing_range=(0.05, 0.1))
    c = mesh.centroids()
    theta = np.arctan2(c[:, 1], c[:, 0])
    assert np.allclose(info[:, 0], p["charge"] * theta)
    assert np.all(info[:, 1] == p["lam_final"]) and np.all(info[:, 2] == 0.5)
    assert not bbar.any() and over["ref_thickness_if_uniform"] == p["thickness"]


def test_build_members_threads(tmp_path):
    """Set-up in threads and meshes from spawned worker processes give the
    same tables."""
    from morphoshell_b200 import ensemble
    a, pa = ensemble.build_members([0, 1, 2], str(tmp_path / "a"), spacing_range=(0.06, 0.1), threads=3)
    b, pb = ensemble.build_members([0, 1, 2], str(tmp_path / "b"), spacing_range=(0.06, 0.1), threads=1,
                                   processes=2)
    for ma, mb in zip(a, b):
        ta, tb = ma.tables(), mb.tables()
        for k in ta:
            assert np.array_equal(ta[k], tb[k]), k
        assert np.array_equal(ma.dofs(1), mb.dofs(1))
    assert pa == pb
